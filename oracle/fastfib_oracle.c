/*
 * fastfib oracle -- TEST INFRASTRUCTURE, not product code.
 *
 * A plain scalar C restatement of the reference's multiply hot path
 * (shwwwa/fastfib): the threshold dispatch, schoolbook / Karatsuba / Toom-3,
 * the three-prime NTT multiply with its width and length choice, Garner CRT
 * with bit packing, the piecewise split multiply, fast doubling and the
 * Barrett decimal conversion.  It restates the algorithm (the same choices,
 * the same integer results); it does not copy the reference's AVX2 code:
 * transforms here are textbook radix-2 / radix-3 loops on `% p` arithmetic.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg call
 * it, and only as the checker.  Parity pin: see fastfib_oracle.h.
 */
#include "fastfib_oracle.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef unsigned __int128 u128;

/* ---------------------------------------------------------------- numbers */

/* Unsigned bignum, little-endian 64-bit limbs, normalized like the
   reference's Big (src/common.h:29-33): n >= 1, top limb nonzero, zero {0}. */
typedef struct {
    uint64_t *d;
    size_t n;
} Num;

static uint64_t g_zero = 0; /* the shared zero of empty views, never freed */

static void *xmal(size_t bytes) {
    void *p = malloc(bytes ? bytes : 8);
    if (!p) {
        fprintf(stderr, "oracle: out of memory (%zu bytes)\n", bytes);
        exit(1);
    }
    return p;
}

static void *xcal(size_t n, size_t s) {
    void *p = calloc(n ? n : 1, s);
    if (!p) {
        fprintf(stderr, "oracle: out of memory (%zu bytes)\n", n * s);
        exit(1);
    }
    return p;
}

/* normalize_len (src/bigint.c:20-23) */
static size_t nlen(const uint64_t *d, size_t n) {
    while (n > 1 && d[n - 1] == 0) n--;
    return n;
}

static void num_free(Num *x) {
    if (x->d && x->d != &g_zero) free(x->d);
    x->d = NULL;
    x->n = 0;
}

static Num num_u64(uint64_t v) {
    Num r = {xmal(8), 1};
    r.d[0] = v;
    return r;
}

static Num num_copy_raw(const uint64_t *d, size_t n) {
    if (n == 0 || d == NULL) return num_u64(0);
    n = nlen(d, n);
    Num r = {xmal(n * 8), n};
    memcpy(r.d, d, n * 8);
    return r;
}

static Num num_copy(const Num *a) { return num_copy_raw(a->d, a->n); }

static int num_is_zero(const Num *a) { return a->n == 1 && a->d[0] == 0; }

/* big_bits (src/bigint.c:44-47); a must be nonzero */
static size_t num_bits(const Num *a) { return 64 * (a->n - 1) + (64 - (size_t)__builtin_clzll(a->d[a->n - 1])); }

/* view_slice (src/bigint.c:50-60): limbs [lo, hi) of a, no copy */
static Num num_view(const Num *a, size_t lo, size_t hi) {
    if (hi > a->n) hi = a->n;
    if (lo >= hi) return (Num){&g_zero, 1};
    return (Num){a->d + lo, nlen(a->d + lo, hi - lo)};
}

/* big_cmp (src/bigint.c:341-347) */
static int num_cmp(const Num *a, const Num *b) {
    if (a->n != b->n) return a->n < b->n ? -1 : 1;
    for (size_t i = a->n; i-- > 0;)
        if (a->d[i] != b->d[i]) return a->d[i] < b->d[i] ? -1 : 1;
    return 0;
}

/* limbs_add_u64 / limbs_sub_u64 (src/bigint.c:69-86) */
static uint64_t ripple_add(uint64_t *d, size_t len, size_t pos, uint64_t v) {
    for (; v && pos < len; pos++) {
        d[pos] += v;
        v = d[pos] < v;
    }
    return v;
}

static uint64_t ripple_sub(uint64_t *d, size_t len, size_t pos, uint64_t v) {
    for (; v && pos < len; pos++) {
        uint64_t old = d[pos];
        d[pos] = old - v;
        v = old < v;
    }
    return v;
}

/* big_add (src/bigint.c:95-106) */
static Num num_add(const Num *a, const Num *b) {
    if (a->n < b->n) {
        const Num *t = a;
        a = b;
        b = t;
    }
    size_t n = a->n + 1;
    uint64_t *d = xmal(n * 8), c = 0;
    for (size_t i = 0; i < a->n; i++) {
        u128 s = (u128)a->d[i] + (i < b->n ? b->d[i] : 0) + c;
        d[i] = (uint64_t)s;
        c = (uint64_t)(s >> 64);
    }
    d[a->n] = c;
    return (Num){d, nlen(d, n)};
}

/* big_sub (src/bigint.c:110-119); requires a >= b */
static Num num_sub(const Num *a, const Num *b) {
    uint64_t *d = xmal(a->n * 8), br = 0;
    for (size_t i = 0; i < a->n; i++) {
        uint64_t y = i < b->n ? b->d[i] : 0;
        u128 t = (u128)a->d[i] - y - br;
        d[i] = (uint64_t)t;
        br = (uint64_t)(t >> 64) ? 1 : 0;
    }
    return (Num){d, nlen(d, a->n)};
}

/* big_add_at (src/bigint.c:124-130): d += x * 2^(64 off) */
static uint64_t add_at(uint64_t *d, size_t dn, const Num *x, size_t off) {
    if (num_is_zero(x)) return 0;
    uint64_t c = 0;
    for (size_t i = 0; i < x->n; i++) {
        u128 s = (u128)d[off + i] + x->d[i] + c;
        d[off + i] = (uint64_t)s;
        c = (uint64_t)(s >> 64);
    }
    return ripple_add(d, dn, off + x->n, c);
}

/* big_sub_at (src/bigint.c:134-140) */
static void sub_at(uint64_t *d, size_t dn, const Num *x, size_t off) {
    if (num_is_zero(x)) return;
    uint64_t br = 0;
    for (size_t i = 0; i < x->n; i++) {
        u128 t = (u128)d[off + i] - x->d[i] - br;
        d[off + i] = (uint64_t)t;
        br = (uint64_t)(t >> 64) ? 1 : 0;
    }
    ripple_sub(d, dn, off + x->n, br);
}

static void num_sub_inplace(Num *x, const Num *y) {
    sub_at(x->d, x->n, y, 0);
    x->n = nlen(x->d, x->n);
}

static void num_add_inplace(Num *x, const Num *y) {
    Num t = num_add(x, y);
    num_free(x);
    *x = t;
}

static void num_add_small(Num *x, uint64_t v) {
    Num t = {&v, 1};
    num_add_inplace(x, &t);
}

static void num_sub_small(Num *x, uint64_t v) {
    Num t = {&v, 1};
    num_sub_inplace(x, &t);
}

/* big_shr_bits (src/bigint.c:203-215) */
static Num num_shr(const Num *a, size_t k) {
    size_t s = k / 64, b = k % 64;
    if (s >= a->n) return num_u64(0);
    size_t n = a->n - s;
    uint64_t *d = xmal(n * 8);
    for (size_t i = 0; i < n; i++) {
        uint64_t lo = a->d[i + s], hi = i + s + 1 < a->n ? a->d[i + s + 1] : 0;
        d[i] = b ? (lo >> b) | (hi << (64 - b)) : lo;
    }
    return (Num){d, nlen(d, n)};
}

/* big_shl_bits (src/bigint.c:220-241) */
static Num num_shl(const Num *a, size_t k) {
    if (num_is_zero(a)) return num_u64(0);
    size_t s = k / 64, b = k % 64, n = a->n + s + 1;
    uint64_t *d = xcal(n, 8), prev = 0;
    for (size_t i = 0; i < a->n; i++) {
        d[i + s] = b ? (a->d[i] << b) | (prev >> (64 - b)) : a->d[i];
        prev = a->d[i];
    }
    d[n - 1] = b ? prev >> (64 - b) : 0;
    return (Num){d, nlen(d, n)};
}

/* big_pow2 (src/bigint.c:244-248) */
static Num num_pow2(size_t k) {
    Num r = {xcal(k / 64 + 1, 8), k / 64 + 1};
    r.d[k / 64] = 1ull << (k % 64);
    return r;
}

/* --------------------------------------------------- schoolbook products */

/* big_mul_schoolbook (src/bigint.c:257-276) */
static Num mul_school(const Num *a, const Num *b) {
    if (num_is_zero(a) || num_is_zero(b)) return num_u64(0);
    size_t n = a->n + b->n;
    uint64_t *d = xcal(n, 8);
    for (size_t i = 0; i < a->n; i++) {
        uint64_t c = 0;
        for (size_t j = 0; j < b->n; j++) {
            u128 t = (u128)a->d[i] * b->d[j] + d[i + j] + c;
            d[i + j] = (uint64_t)t;
            c = (uint64_t)(t >> 64);
        }
        d[i + b->n] = c;
    }
    return (Num){d, nlen(d, n)};
}

/* ------------------------------------------------------- NTT definitions */

static int MAX_LG = 25; /* NTT_MAX_LG (src/common.h:46-48); fo_set_max_lg mirrors -DNTT_MAX_LG */
static const uint32_t P[3] = {2113929217u, 2013265921u, 1811939329u}; /* src/ntt_arith.c:48-52 */
static const uint32_t G[3] = {5, 31, 13};

static size_t g_max_L = 0; /* g_ntt_max_L (src/mul_basic.c:26) */

static uint32_t pw(uint32_t a, uint64_t e, uint32_t p) {
    uint64_t r = 1, x = a % p;
    for (; e; e >>= 1, x = x * x % p)
        if (e & 1) r = r * x % p;
    return (uint32_t)r;
}

static inline uint32_t mm(uint32_t a, uint32_t b, uint32_t p) { return (uint32_t)((uint64_t)a * b % p); }
static inline uint32_t ad(uint32_t a, uint32_t b, uint32_t p) { uint32_t s = a + b; return s >= p ? s - p : s; }
static inline uint32_t sb(uint32_t a, uint32_t b, uint32_t p) { return a >= b ? a - b : a + p - b; }

/* ntt_init (src/ntt_tables.c:72-75, 123): the tables only grow */
void fo_ntt_init(size_t max_limbs) {
    size_t L = 16;
    while (L < 2 * max_limbs && L < ((size_t)1 << MAX_LG)) L <<= 1;
    if (L > g_max_L) g_max_L = L;
}
size_t fo_ntt_max_L(void) { return g_max_L; }
void fo_set_max_lg(int lg) {
    MAX_LG = lg;
    if (g_max_L > ((size_t)1 << lg)) g_max_L = (size_t)1 << lg;
}
void fo_set_ntt_max_L(size_t L) { g_max_L = L; }

/* ntt_width_ok (src/mul_ntt.c:55-59) */
static int width_ok(uint64_t bits_a, uint64_t bits_b, unsigned w) {
    const u128 M = (u128)P[0] * P[1] * P[2];
    uint64_t ca = (bits_a + w - 1) / w, cb = (bits_b + w - 1) / w;
    return ((u128)(ca < cb ? ca : cb) << (2 * w)) < M;
}

/* ntt_length (src/mul_ntt.c:78-93) */
static uint64_t ntt_len(uint64_t conv, uint32_t *lg_out, uint32_t *r3_out) {
    uint64_t L = 16;
    uint32_t lg = 4, r3 = 0;
    while (L < conv) {
        L <<= 1;
        lg++;
    }
    if (L / 4 * 3 >= conv && L / 4 >= 16) {
        L = L / 4 * 3;
        lg -= 2;
        r3 = 1;
    }
    *lg_out = lg;
    *r3_out = r3;
    return L;
}

/* The split's width and piece length (src/mul_split.c:150-177). */
static void split_plan(uint64_t bits_a, uint64_t bits_b, int square, FoPlan *pl) {
    unsigned bw = 35;
    while (bw > 8 && !width_ok(bits_a, bits_b, bw)) bw--;
    size_t cap = g_max_L < ((size_t)1 << MAX_LG) ? g_max_L : ((size_t)1 << MAX_LG);
    if (cap < 16) cap = 16; /* no tables yet: the smallest ntt_init builds 16 */
    int lgmax = __builtin_ctzll(cap);
    int lgp = lgmax;
    double best = 0;
    for (int lg = lgmax; lg >= lgmax - 4 && lg >= 10; lg--) {
        uint64_t h = (uint64_t)1 << (lg - 1);
        uint64_t ka = ((bits_a + bw - 1) / bw + h - 1) / h, kb = ((bits_b + bw - 1) / bw + h - 1) / h;
        double ca = (double)ka, cb = (double)kb;
        double tr = square ? 3 * ca - 1 : 2 * (ca + cb) - 1, pairs = square ? ca * (ca + 1) / 2 : ca * cb;
        double cost = (tr * lg + 5 * pairs) * (double)((uint64_t)1 << lg);
        if (lg == lgmax || cost < best) best = cost, lgp = lg;
    }
    uint64_t Lp = (uint64_t)1 << lgp, H = Lp / 2;
    memset(pl, 0, sizeof *pl);
    pl->split = 1;
    pl->width = bw;
    pl->lg = (uint32_t)lgp;
    pl->L = Lp;
    pl->ca = (bits_a + bw - 1) / bw;
    pl->cb = (bits_b + bw - 1) / bw;
    pl->ka = (pl->ca + H - 1) / H;
    pl->kb = square ? pl->ka : (pl->cb + H - 1) / H;
    pl->conv = pl->ca + pl->cb - 1;
    pl->Lbig = (pl->ka + pl->kb) * H;
}

/* big_mul_ntt's choice (src/mul_ntt.c:97-118): the shortest transform over
   widths 32..35 that pass the CRT bound, the narrowest among equals; the
   split when none fits or the transform is past the tables. Returns split. */
int fo_ntt_plan(uint64_t bits_a, uint64_t bits_b, int square, FoPlan *pl) {
    memset(pl, 0, sizeof *pl);
    uint64_t L = 0;
    for (unsigned w = 32; w <= 35; w++) {
        if (!width_ok(bits_a, bits_b, w)) break;
        uint64_t ca = (bits_a + w - 1) / w, cb = (bits_b + w - 1) / w;
        uint32_t lg, r3;
        uint64_t Lw = ntt_len(ca + cb - 1, &lg, &r3);
        if (L == 0 || Lw < L) {
            L = Lw;
            pl->L = Lw, pl->lg = lg, pl->r3 = r3, pl->width = w;
            pl->ca = ca, pl->cb = cb, pl->conv = ca + cb - 1;
        }
    }
    if (L == 0 || L > g_max_L) {
        split_plan(bits_a, bits_b, square, pl);
        return 1;
    }
    return 0;
}

/* ------------------------------------------------------------ transforms */

/* Forward DFT of length L = 2^k or 3 * 2^k mod p, in place, natural order in
   and out: X[k] = sum_n x[n] w^(nk), w a primitive L-th root of unity.  The
   radix-2 part is the textbook iterative Cooley-Tukey; a 3 * 2^k length runs
   three 2^k transforms on the interleaved thirds x[3m + t] and combines them
   with X[k] = sum_t w^(tk) Y_t[k mod 2^k]. `inv` uses w^-1 (no 1/L here). */
static void dft2(uint32_t *a, uint64_t n, uint32_t w, uint32_t p) {
    for (uint64_t i = 1, j = 0; i < n; i++) {
        uint64_t bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) {
            uint32_t t = a[i];
            a[i] = a[j];
            a[j] = t;
        }
    }
    uint32_t *tw = xmal(n / 2 * 4 + 4);
    for (uint64_t len = 2; len <= n; len <<= 1) {
        uint32_t wl = pw(w, n / len, p);
        tw[0] = 1;
        for (uint64_t j = 1; j < len / 2; j++) tw[j] = mm(tw[j - 1], wl, p);
        for (uint64_t i = 0; i < n; i += len)
            for (uint64_t j = 0; j < len / 2; j++) {
                uint32_t u = a[i + j], v = mm(a[i + j + len / 2], tw[j], p);
                a[i + j] = ad(u, v, p);
                a[i + j + len / 2] = sb(u, v, p);
            }
    }
    free(tw);
}

static void dft(uint32_t *a, uint64_t L, int inv, uint32_t p, uint32_t g) {
    uint32_t w = pw(g, (p - 1) / L, p);
    if (inv) w = pw(w, p - 2, p);
    if ((L & (L - 1)) == 0) {
        dft2(a, L, w, p);
        return;
    }
    uint64_t M = L / 3;
    uint32_t *y = xmal(L * 4);
    for (int t = 0; t < 3; t++) {
        for (uint64_t m = 0; m < M; m++) y[t * M + m] = a[3 * m + t];
        dft2(y + t * M, M, pw(w, 3, p), p);
    }
    uint32_t wk = 1;
    for (uint64_t k = 0; k < L; k++, wk = mm(wk, w, p)) {
        uint32_t s = y[k % M];
        s = ad(s, mm(wk, y[M + k % M], p), p);
        s = ad(s, mm(mm(wk, wk, p), y[2 * M + k % M], p), p);
        a[k] = s;
    }
    free(y);
}

/* Coefficient i of a as a b-bit digit: bits [i b, i b + b) (the Src reader,
   src/ntt_kernels.c:29-74), zero past the end. */
static uint64_t digit(const Num *a, uint64_t i, unsigned b) {
    uint64_t bit = i * b, q = bit / 64, off = bit % 64;
    if (q >= a->n) return 0;
    u128 w = a->d[q];
    if (q + 1 < a->n) w |= (u128)a->d[q + 1] << 64;
    return (uint64_t)(w >> off) & (((uint64_t)1 << b) - 1);
}

/* The three residues of every coefficient of the product -> the integer:
   Garner's method X = x1 + x2 p1 + x3 p1 p2 (src/crt.c:38-64), then X added
   at bit i b with a running carry (src/crt.c:70-87, 105-150). */
static Num crt_pack(uint32_t *const y[3], uint64_t conv, unsigned b, size_t limbs) {
    const uint32_t p1 = P[0], p2 = P[1], p3 = P[2];
    const uint32_t i12 = pw(p1 % p2, p2 - 2, p2), i13 = pw(p1 % p3, p3 - 2, p3), i23 = pw(p2 % p3, p3 - 2, p3);
    uint64_t *d = xcal(limbs, 8);
    u128 c = 0, mask = ((u128)1 << b) - 1;
    for (uint64_t i = 0; i < conv; i++) {
        uint32_t r1 = y[0][i], r2 = y[1][i], r3 = y[2][i];
        uint32_t x2 = mm(sb(r2, r1 % p2, p2), i12, p2);
        uint32_t t3 = mm(sb(r3, r1 % p3, p3), i13, p3);
        uint32_t x3 = mm(sb(t3, x2 % p3, p3), i23, p3);
        u128 X = (u128)r1 + (u128)x2 * p1 + (u128)x3 * ((u128)p1 * p2);
        u128 acc = X + c;
        uint64_t v = (uint64_t)(acc & mask);
        c = acc >> b;
        uint64_t bit = i * b, q = bit / 64, off = bit % 64;
        if (q < limbs) d[q] |= v << off;
        if (off + b > 64 && q + 1 < limbs) d[q + 1] |= v >> (64 - off);
    }
    /* the final carry lands at bit conv * b */
    uint64_t bit = conv * b, q = bit / 64, off = bit % 64;
    for (; c && q < limbs; q++) {
        u128 s = (u128)d[q] + (uint64_t)(c << off);
        d[q] = (uint64_t)s;
        c = (c >> (64 - off)) + (s >> 64);
        off = 0;
    }
    return (Num){d, nlen(d, limbs)};
}

/* One prime's cyclic convolution of the width-w digits of a and b at length
   L, scaled by 1/L (src/mul_ntt.c:29-48): L words, malloc'd. */
static uint32_t *conv_prime(const Num *a, const Num *b, int square, unsigned w, uint64_t L, int k) {
    uint64_t ca = (num_bits(a) + w - 1) / w, cb = (num_bits(b) + w - 1) / w;
    uint32_t p = P[k];
    uint32_t *fa = xcal(L, 4), *fb = square ? fa : xcal(L, 4);
    for (uint64_t i = 0; i < ca; i++) fa[i] = (uint32_t)(digit(a, i, w) % p);
    if (!square)
        for (uint64_t i = 0; i < cb; i++) fb[i] = (uint32_t)(digit(b, i, w) % p);
    dft(fa, L, 0, p, G[k]);
    if (!square) dft(fb, L, 0, p, G[k]);
    for (uint64_t i = 0; i < L; i++) fa[i] = mm(fa[i], fb[i], p);
    dft(fa, L, 1, p, G[k]);
    uint32_t linv = pw((uint32_t)(L % p), p - 2, p);
    for (uint64_t i = 0; i < L; i++) fa[i] = mm(fa[i], linv, p);
    if (!square) free(fb);
    return fa;
}

/* big_mul_ntt for a given width and transform length: three cyclic
   convolutions, then the CRT (src/mul_ntt.c:65-73). */
static Num mul_ntt_plain(const Num *a, const Num *b, int square, unsigned w, uint64_t L) {
    size_t bits_a = num_bits(a), bits_b = num_bits(b);
    uint64_t ca = (bits_a + w - 1) / w, cb = (bits_b + w - 1) / w, conv = ca + cb - 1;
    uint32_t *y[3];
    for (int k = 0; k < 3; k++) y[k] = conv_prime(a, b, square, w, L, k);
    Num r = crt_pack(y, conv, w, a->n + b->n + 1);
    for (int k = 0; k < 3; k++) free(y[k]);
    return r;
}

/* big_mul_ntt_split (src/mul_split.c:98-187): pieces of H = Lp/2
   coefficients transformed once; output piece m = sum_{i+j=m} A_i B_j in the
   transform domain, one inverse per m, overlap-added at m H; then the CRT. */
static Num mul_split(const Num *a, const Num *b, int square, const FoPlan *pl) {
    const uint64_t Lp = pl->L, H = Lp / 2, ka = pl->ka, kb = pl->kb;
    const unsigned w = pl->width;
    uint32_t *y[3];
    for (int k = 0; k < 3; k++) {
        uint32_t p = P[k];
        uint32_t *A = xcal(ka * Lp, 4), *B = square ? A : xcal(kb * Lp, 4);
        for (uint64_t i = 0; i < ka; i++) {
            for (uint64_t t = 0; t < H && i * H + t < pl->ca; t++) A[i * Lp + t] = (uint32_t)(digit(a, i * H + t, w) % p);
            dft(A + i * Lp, Lp, 0, p, G[k]);
        }
        if (!square)
            for (uint64_t j = 0; j < kb; j++) {
                for (uint64_t t = 0; t < H && j * H + t < pl->cb; t++) B[j * Lp + t] = (uint32_t)(digit(b, j * H + t, w) % p);
                dft(B + j * Lp, Lp, 0, p, G[k]);
            }
        uint32_t *Y = xcal(pl->Lbig + Lp, 4), *C = xmal(Lp * 4);
        uint32_t linv = pw((uint32_t)(Lp % p), p - 2, p);
        for (uint64_t m = 0; m + 1 < ka + kb; m++) {
            uint64_t i0 = m + 1 > kb ? m + 1 - kb : 0, i1 = m < ka - 1 ? m : ka - 1;
            memset(C, 0, Lp * 4);
            for (uint64_t i = i0; i <= i1; i++)
                for (uint64_t x = 0; x < Lp; x++) C[x] = ad(C[x], mm(A[i * Lp + x], B[(m - i) * Lp + x], p), p);
            dft(C, Lp, 1, p, G[k]);
            for (uint64_t t = 0; t < Lp; t++) Y[m * H + t] = ad(Y[m * H + t], mm(C[t], linv, p), p);
        }
        free(C);
        if (!square) free(B);
        free(A);
        y[k] = Y;
    }
    Num r = crt_pack(y, pl->conv, w, a->n + b->n + 1);
    for (int k = 0; k < 3; k++) free(y[k]);
    return r;
}

/* big_mul_ntt (src/mul_ntt.c:97-142) */
static Num mul_ntt(const Num *a, const Num *b, int square) {
    if (num_is_zero(a) || num_is_zero(b)) return num_u64(0);
    FoPlan pl;
    if (fo_ntt_plan(num_bits(a), num_bits(b), square, &pl)) return mul_split(a, b, square, &pl);
    return mul_ntt_plain(a, b, square, pl.width, pl.L);
}

/* ------------------------------------------------------ the dispatch (L5) */

#define KARATSUBA_THRESHOLD_LIMBS 64 /* src/mul_basic.c:30-38 */
#define NTT_THRESHOLD_LIMBS 200
#define TOOM3_THRESHOLD_LIMBS 1500

static Num mul_any(const Num *a, const Num *b);
static Num sqr_any(const Num *a);

/* ntt_fits (src/mul_basic.c:41-43) */
static int ntt_fits(const Num *a, const Num *b) {
    return 2 * (a->n + b->n) - 1 <= g_max_L || g_max_L >= ((size_t)1 << MAX_LG);
}

/* karatsuba_combine (src/mul_basic.c:46-61) */
static Num kara_combine(Num *z0, Num *z1, Num *z2, size_t half, size_t n) {
    sub_at(z1->d, z1->n, z2, 0);
    sub_at(z1->d, z1->n, z0, 0);
    z1->n = nlen(z1->d, z1->n);
    uint64_t *d = xcal(n, 8);
    add_at(d, n, z0, 0);
    add_at(d, n, z1, half);
    add_at(d, n, z2, 2 * half);
    num_free(z0);
    num_free(z1);
    num_free(z2);
    return (Num){d, nlen(d, n)};
}

/* Signed numbers for Toom-3 (src/bigint.c:353-407) */
typedef struct {
    int neg;
    Num mag;
} SNum;

static SNum s_wrap(Num m, int neg) { return (SNum){num_is_zero(&m) ? 0 : neg, m}; }
static SNum s_add(const SNum *x, const SNum *y) {
    if (x->neg == y->neg) return s_wrap(num_add(&x->mag, &y->mag), x->neg);
    int c = num_cmp(&x->mag, &y->mag);
    if (c == 0) return s_wrap(num_u64(0), 0);
    return c > 0 ? s_wrap(num_sub(&x->mag, &y->mag), x->neg) : s_wrap(num_sub(&y->mag, &x->mag), y->neg);
}
static SNum s_sub(const SNum *x, const SNum *y) {
    SNum ny = {num_is_zero(&y->mag) ? 0 : !y->neg, y->mag};
    return s_add(x, &ny);
}
static SNum s_diff(const Num *x, const Num *y) {
    return num_cmp(x, y) >= 0 ? s_wrap(num_sub(x, y), 0) : s_wrap(num_sub(y, x), 1);
}
/* exact division by 2 or 3 (big_divmod_small_inplace, src/bigint.c:327-337) */
static SNum s_div(const SNum *x, uint32_t dv) {
    Num t = num_copy(&x->mag);
    u128 rem = 0;
    for (size_t i = t.n; i-- > 0;) {
        u128 cur = (rem << 64) | t.d[i];
        t.d[i] = (uint64_t)(cur / dv);
        rem = cur % dv;
    }
    t.n = nlen(t.d, t.n);
    return s_wrap(t, x->neg);
}
static void s_free(SNum *x) { num_free(&x->mag); }

/* big_mul_toom3 (src/mul_basic.c:175-252): 5-point Toom-Cook at 0, 1, -1, -2, inf */
static Num mul_toom3(const Num *a, const Num *b, int sq) {
    size_t maxlen = a->n > b->n ? a->n : b->n, k = (maxlen + 2) / 3;
    Num x[3] = {num_view(a, 0, k), num_view(a, k, 2 * k), num_view(a, 2 * k, a->n)};
    Num y[3] = {num_view(b, 0, k), num_view(b, k, 2 * k), num_view(b, 2 * k, b->n)};
    Num e1[2];
    SNum em1[2], em2[2];
    for (int s = 0; s < (sq ? 1 : 2); s++) {
        Num *v = s ? y : x;
        Num t = num_add(&v[0], &v[2]);
        e1[s] = num_add(&t, &v[1]);
        em1[s] = s_diff(&t, &v[1]);
        num_free(&t);
        Num x24 = num_shl(&v[2], 2), x12 = num_shl(&v[1], 1), s04 = num_add(&v[0], &x24);
        em2[s] = s_diff(&s04, &x12);
        num_free(&x24);
        num_free(&x12);
        num_free(&s04);
    }
    int o = sq ? 0 : 1;
#define TMUL(u, v) (sq ? sqr_any(u) : mul_any(u, v))
    Num R0m = TMUL(&x[0], &y[0]), Rim = TMUL(&x[2], &y[2]), R1m = TMUL(&e1[0], &e1[o]);
    SNum Rm1 = s_wrap(TMUL(&em1[0].mag, &em1[o].mag), em1[0].neg ^ em1[o].neg);
    SNum Rm2 = s_wrap(TMUL(&em2[0].mag, &em2[o].mag), em2[0].neg ^ em2[o].neg);
#undef TMUL
    for (int s = 0; s < (sq ? 1 : 2); s++) {
        num_free(&e1[s]);
        s_free(&em1[s]);
        s_free(&em2[s]);
    }
    SNum R0 = s_wrap(R0m, 0), R1 = s_wrap(R1m, 0), Ri = s_wrap(Rim, 0);
    SNum t = s_sub(&Rm2, &R1), r3 = s_div(&t, 3);
    s_free(&t);
    t = s_sub(&R1, &Rm1);
    SNum r1 = s_div(&t, 2);
    s_free(&t);
    SNum r2 = s_sub(&Rm1, &R0);
    s_free(&Rm1);
    s_free(&Rm2);
    s_free(&R1);
    t = s_sub(&r2, &r3);
    SNum h = s_div(&t, 2);
    s_free(&t);
    s_free(&r3);
    SNum ri2 = s_wrap(num_shl(&Ri.mag, 1), 0);
    r3 = s_add(&h, &ri2);
    s_free(&h);
    s_free(&ri2);
    t = s_add(&r2, &r1);
    s_free(&r2);
    r2 = s_sub(&t, &Ri);
    s_free(&t);
    t = s_sub(&r1, &r3);
    s_free(&r1);
    r1 = t;
    size_t n = a->n + b->n;
    uint64_t *d = xcal(n, 8);
    add_at(d, n, &R0.mag, 0);
    add_at(d, n, &r1.mag, k);
    add_at(d, n, &r2.mag, 2 * k);
    add_at(d, n, &r3.mag, 3 * k);
    add_at(d, n, &Ri.mag, 4 * k);
    s_free(&R0);
    s_free(&r1);
    s_free(&r2);
    s_free(&r3);
    s_free(&Ri);
    return (Num){d, nlen(d, n)};
}

/* big_mul (src/mul_basic.c:64-106) */
static Num mul_any(const Num *a, const Num *b) {
    size_t minlen = a->n < b->n ? a->n : b->n;
    if (minlen <= KARATSUBA_THRESHOLD_LIMBS) return mul_school(a, b);
    if (minlen >= NTT_THRESHOLD_LIMBS && ntt_fits(a, b)) return mul_ntt(a, b, a == b);
    if (minlen >= TOOM3_THRESHOLD_LIMBS) return mul_toom3(a, b, 0);
    size_t half = (a->n > b->n ? a->n : b->n) / 2;
    Num al = num_view(a, 0, half), ah = num_view(a, half, a->n);
    Num bl = num_view(b, 0, half), bh = num_view(b, half, b->n);
    Num z0 = mul_any(&al, &bl), z2 = mul_any(&ah, &bh);
    Num sa = num_add(&al, &ah), sbb = num_add(&bl, &bh);
    Num z1 = mul_any(&sa, &sbb);
    num_free(&sa);
    num_free(&sbb);
    return kara_combine(&z0, &z1, &z2, half, a->n + b->n);
}

/* big_sqr (src/mul_basic.c:109-132); a plain product stands in for the
   schoolbook square (same integer). */
static Num sqr_any(const Num *a) {
    if (a->n <= KARATSUBA_THRESHOLD_LIMBS) return mul_school(a, a);
    if (a->n >= NTT_THRESHOLD_LIMBS && ntt_fits(a, a)) return mul_ntt(a, a, 1);
    if (a->n >= TOOM3_THRESHOLD_LIMBS) return mul_toom3(a, a, 1);
    size_t half = a->n / 2;
    Num al = num_view(a, 0, half), ah = num_view(a, half, a->n);
    Num z0 = sqr_any(&al), z2 = sqr_any(&ah);
    Num sa = num_add(&al, &ah);
    Num z1 = sqr_any(&sa);
    num_free(&sa);
    return kara_combine(&z0, &z1, &z2, half, 2 * a->n);
}

/* ------------------------------------------------------- fast doubling */

#define LOG2_PHI 0.6942419136306174 /* src/fib.c:200 */

/* fib_step_linear (src/fib.c:19-109): from s1 = F(k)^2, s2 = F(k-1)^2,
   A = s1 + s2 = F(2k-1), B = 4 s1 - s2 + 2(-1)^k = F(2k+1), C = B - A. */
static void fib_step(const Num *s1, const Num *s2, int k_odd, int bit, Num *lo, Num *hi) {
    Num A = num_add(s1, s2);
    Num s4 = num_shl(s1, 2);
    Num B = num_sub(&s4, s2);
    num_free(&s4);
    if (k_odd) num_sub_small(&B, 2);
    else num_add_small(&B, 2);
    Num C = num_sub(&B, &A);
    if (bit) {
        *lo = C;
        *hi = B;
        num_free(&A);
    } else {
        *lo = A;
        *hi = C;
        num_free(&B);
    }
}

/* fibonacci (src/fib.c:211-261) */
static Num fib(uint64_t n) {
    if (n == 0) return num_u64(0);
    fo_ntt_init((size_t)((double)n * LOG2_PHI / 64.0) + 8);
    Num fkm1 = num_u64(0), fk = num_u64(1);
    int k_odd = 1, top = 63 - __builtin_clzll(n);
    for (int i = top - 1; i >= 1; i--) {
        Num s1 = sqr_any(&fk), s2 = sqr_any(&fkm1);
        num_free(&fkm1);
        num_free(&fk);
        int bit = (int)((n >> i) & 1);
        fib_step(&s1, &s2, k_odd, bit, &fkm1, &fk);
        num_free(&s1);
        num_free(&s2);
        k_odd = bit;
    }
    if (top == 0) {
        num_free(&fkm1);
        return fk;
    }
    Num result;
    if (n & 1) { /* (2F(k) + F(k-1)) (2F(k) - F(k-1)) + 2(-1)^k, src/fib.c:239-250 */
        Num u2 = num_shl(&fk, 1);
        Num x = num_add(&u2, &fkm1), y = num_sub(&u2, &fkm1);
        num_free(&u2);
        num_free(&fk);
        num_free(&fkm1);
        result = mul_any(&x, &y);
        num_free(&x);
        num_free(&y);
        if (k_odd) num_sub_small(&result, 2);
        else num_add_small(&result, 2);
    } else { /* F(k) (F(k) + 2F(k-1)), src/fib.c:251-258 */
        Num v2 = num_shl(&fkm1, 1);
        Num x = num_add(&fk, &v2);
        num_free(&v2);
        num_free(&fkm1);
        result = mul_any(&fk, &x);
        num_free(&x);
        num_free(&fk);
    }
    return result;
}

/* ----------------------------------------------------------- decimal */

#define DEC_LEAF_LG 4 /* src/decimal.c:24-27 */
#define DEC_P0 10000000000000000000ull

/* big_recip (src/decimal.c:39-71): floor(2^(2s)/P) minus at most 4 */
static Num recip(const Num *Pn, size_t s) {
    if (s <= 62) return num_u64((uint64_t)(((u128)1 << (2 * s)) / Pn->d[0]));
    size_t h = (s + 1) / 2 + 16;
    Num Ph = num_shr(Pn, s - h), mh = recip(&Ph, h);
    num_free(&Ph);
    Num y = num_shl(&mh, s - h);
    num_free(&mh);
    Num Z = num_pow2(2 * s), d = mul_any(Pn, &y);
    int below = num_cmp(&d, &Z) <= 0;
    Num e = below ? num_sub(&Z, &d) : num_sub(&d, &Z);
    num_free(&d);
    Num ye = mul_any(&y, &e);
    num_free(&e);
    Num corr = num_shr(&ye, 2 * s);
    num_free(&ye);
    if (below) num_add_inplace(&y, &corr);
    else num_sub_inplace(&y, &corr);
    num_free(&corr);
    num_free(&Z);
    num_sub_small(&y, 2);
    return y;
}

/* big_divmod_barrett (src/decimal.c:76-89) */
static void divmod_barrett(const Num *x, const Num *Pn, const Num *m, size_t s, Num *q, Num *r) {
    Num q1 = num_shr(x, s - 1), t = mul_any(&q1, m);
    num_free(&q1);
    *q = num_shr(&t, s + 1);
    num_free(&t);
    Num qp = mul_any(q, Pn);
    *r = num_sub(x, &qp);
    num_free(&qp);
    while (num_cmp(r, Pn) >= 0) {
        num_sub_inplace(r, Pn);
        num_add_small(q, 1);
    }
}

/* big_divmod_any (src/decimal.c:95-125) */
static void divmod_any(const Num *x, const Num *Pn, size_t s, Num *q, Num *r) {
    size_t bx = num_is_zero(x) ? 0 : num_bits(x);
    if (bx < s) {
        *q = num_u64(0);
        *r = num_copy(x);
        return;
    }
    size_t t = bx - s + 1, k = t + 64 < s ? t + 64 : s;
    Num Pk = num_shr(Pn, s - k), Xk = num_shr(x, s - k), mk = recip(&Pk, k), rk;
    divmod_barrett(&Xk, &Pk, &mk, k, q, &rk);
    num_free(&Pk);
    num_free(&Xk);
    num_free(&mk);
    num_free(&rk);
    Num qp = mul_any(q, Pn);
    while (num_cmp(&qp, x) > 0) {
        num_sub_small(q, 1);
        num_sub_inplace(&qp, Pn);
    }
    *r = num_sub(x, &qp);
    num_free(&qp);
    while (num_cmp(r, Pn) >= 0) {
        num_sub_inplace(r, Pn);
        num_add_small(q, 1);
    }
}

/* dec_leaf (src/decimal.c:139-150): 19 * chunks digits by repeated division by 10^19 */
static void dec_leaf(const Num *x, size_t chunks, char *out) {
    size_t n = x->n;
    uint64_t *t = xmal(n * 8);
    memcpy(t, x->d, n * 8);
    for (size_t c = chunks; c-- > 0;) {
        uint64_t rem = 0;
        for (size_t i = n; i-- > 0;) {
            u128 cur = ((u128)rem << 64) | t[i];
            t[i] = (uint64_t)(cur / DEC_P0);
            rem = (uint64_t)(cur % DEC_P0);
        }
        while (n > 1 && t[n - 1] == 0) n--;
        char *o = out + 19 * c;
        for (int j = 18; j >= 0; j--, rem /= 10) o[j] = (char)('0' + rem % 10);
    }
    free(t);
}

typedef struct {
    Num pw[48], inv[48];
    size_t bits[48];
} DecCtx;

/* dec_emit (src/decimal.c:192-203): 2 * 19 * 2^lvl digits of x < P_lvl^2 */
static void dec_emit(const DecCtx *c, Num x, int lvl, char *out) {
    if (lvl <= DEC_LEAF_LG) {
        dec_leaf(&x, (size_t)2 << lvl, out);
        num_free(&x);
        return;
    }
    Num q, r;
    divmod_barrett(&x, &c->pw[lvl], &c->inv[lvl], c->bits[lvl], &q, &r);
    num_free(&x);
    dec_emit(c, q, lvl - 1, out);
    dec_emit(c, r, lvl - 1, out + ((size_t)19 << lvl));
}

/* big_to_string (src/decimal.c:229-281) */
static char *to_string(const Num *a) {
    if (num_is_zero(a)) {
        char *s = xmal(2);
        s[0] = '0';
        s[1] = 0;
        return s;
    }
    static DecCtx c; /* large; the oracle is single-threaded */
    size_t ba = num_bits(a);
    int T = 0;
    c.pw[0] = num_u64(DEC_P0);
    c.bits[0] = num_bits(&c.pw[0]);
    while (2 * (c.bits[T] - 1) < ba) {
        c.pw[T + 1] = sqr_any(&c.pw[T]);
        c.bits[T + 1] = num_bits(&c.pw[T + 1]);
        T++;
    }
    for (int i = DEC_LEAF_LG + 1; i < T; i++) c.inv[i] = recip(&c.pw[i], c.bits[i]);
    size_t half = (size_t)19 << T, total = 2 * half;
    char *buf = xmal(total + 1);
    if (T <= DEC_LEAF_LG) {
        dec_leaf(a, (size_t)2 << T, buf);
    } else {
        Num q, r;
        divmod_any(a, &c.pw[T], c.bits[T], &q, &r);
        dec_emit(&c, q, T - 1, buf);
        dec_emit(&c, r, T - 1, buf + half);
    }
    for (int i = 0; i <= T; i++) num_free(&c.pw[i]);
    for (int i = DEC_LEAF_LG + 1; i < T; i++) num_free(&c.inv[i]);
    size_t z = 0;
    while (z + 1 < total && buf[z] == '0') z++;
    memmove(buf, buf + z, total - z);
    buf[total - z] = 0;
    return buf;
}

/* ---------------------------------------------------------- exported API */

static uint64_t *take(Num *r, size_t *nout) {
    uint64_t *o = xmal(r->n * 8);
    memcpy(o, r->d, r->n * 8);
    *nout = r->n;
    num_free(r);
    return o;
}

uint64_t *fo_mul(const uint64_t *a, size_t na, const uint64_t *b, size_t nb, int square, size_t *nout) {
    Num A = num_copy_raw(a, na), B = square ? A : num_copy_raw(b, nb);
    Num r = square ? sqr_any(&A) : mul_any(&A, &B);
    num_free(&A);
    if (!square) num_free(&B);
    return take(&r, nout);
}

uint64_t *fo_mul_ntt(const uint64_t *a, size_t na, const uint64_t *b, size_t nb, int square, size_t *nout) {
    Num A = num_copy_raw(a, na), B = square ? A : num_copy_raw(b, nb);
    Num r = mul_ntt(&A, &B, square);
    num_free(&A);
    if (!square) num_free(&B);
    return take(&r, nout);
}

/* One NTT product at a caller-chosen width and transform length (the
   forced-plan mode of the microbench); L must hold the product's
   coefficients and divide 3 * 2^25. */
uint64_t *fo_mul_ntt_forced(const uint64_t *a, size_t na, const uint64_t *b, size_t nb, int square,
                            uint32_t width, uint64_t L, size_t *nout) {
    Num A = num_copy_raw(a, na), B = square ? A : num_copy_raw(b, nb);
    Num r = (num_is_zero(&A) || num_is_zero(&B)) ? num_u64(0) : mul_ntt_plain(&A, &B, square, width, L);
    num_free(&A);
    if (!square) num_free(&B);
    return take(&r, nout);
}

/* One prime's share of a product sharded by prime: the scaled convolution
   modulo prime k (0..2) at width and length L into y[0 .. L); -1 when L does
   not hold the product's coefficients. */
int fo_residues(const uint64_t *a, size_t na, const uint64_t *b, size_t nb, int square, uint32_t width,
                uint64_t L, int k, uint32_t *y) {
    Num A = num_copy_raw(a, na), B = square ? A : num_copy_raw(b, nb);
    const uint64_t ca = (num_bits(&A) + width - 1) / width, cb = (num_bits(&B) + width - 1) / width;
    if (k < 0 || k > 2 || width < 1 || width > 35 || ca + cb - 1 > L) {
        num_free(&A);
        if (!square) num_free(&B);
        return -1;
    }
    uint32_t *f = conv_prime(&A, &B, square, width, L, k);
    memcpy(y, f, L * 4);
    free(f);
    num_free(&A);
    if (!square) num_free(&B);
    return 0;
}

/* The product from all three primes' residues (y: 3 * L words, prime-major),
   conv coefficients of width bits, limbs limbs at most. */
uint64_t *fo_crt_residues(const uint32_t *y, uint64_t L, uint64_t conv, uint32_t width, size_t limbs,
                          size_t *nout) {
    uint32_t *const ys[3] = {(uint32_t *)y, (uint32_t *)y + L, (uint32_t *)y + 2 * L};
    Num r = crt_pack(ys, conv, width, limbs);
    return take(&r, nout);
}

uint64_t *fo_fibonacci(uint64_t n, size_t *nout) {
    Num r = fib(n);
    return take(&r, nout);
}

char *fo_to_string(const uint64_t *a, size_t na) {
    Num A = num_copy_raw(a, na);
    char *s = to_string(&A);
    num_free(&A);
    return s;
}

/* The fingerprint of tests/memrun.c:19-27: bits, low 64 bits, and the value
   mod four 64-bit primes. */
void fo_fingerprint(const uint64_t *a, size_t na, uint64_t out[6]) {
    static const uint64_t ps[4] = {18446744073709551557ull, 18446744073709551533ull, 9223372036854775783ull,
                                   4611686018427387847ull};
    Num A = {(uint64_t *)a, na ? nlen(a, na) : 0};
    out[0] = (A.n == 0 || num_is_zero(&A)) ? 0 : num_bits(&A);
    out[1] = A.n ? A.d[0] : 0;
    for (int i = 0; i < 4; i++) {
        u128 m = 0;
        for (size_t k = A.n; k-- > 0;) m = ((m << 64) | A.d[k]) % ps[i];
        out[2 + i] = (uint64_t)m;
    }
}

void fo_free(void *p) { free(p); }
