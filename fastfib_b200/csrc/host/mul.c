/*
 * The multiply dispatch of the reference's surface (src/mul_basic.c:64-132):
 * schoolbook up to KARATSUBA_THRESHOLD_LIMBS, the NTT from
 * NTT_THRESHOLD_LIMBS when the transform cap allows it (ntt_fits), Toom-3
 * past TOOM3_THRESHOLD_LIMBS otherwise, Karatsuba between.  The thresholds
 * are the reference's (overridable with -D like there).  big_mul_ntt runs on
 * the GPU through ffg_mul_host; squaring is signalled by a == b.
 */
#include <string.h>

#include "fastfib.h"
#include "ffg.h"
#include "host_internal.h"

#ifndef KARATSUBA_THRESHOLD_LIMBS
#define KARATSUBA_THRESHOLD_LIMBS 64
#endif
#ifndef NTT_THRESHOLD_LIMBS
#define NTT_THRESHOLD_LIMBS 200
#endif
#ifndef TOOM3_THRESHOLD_LIMBS
#define TOOM3_THRESHOLD_LIMBS 1500
#endif
#define NTT_MAX_LG 25

size_t g_ntt_max_L = 0;

void ntt_init(size_t max_limbs) {
    int rc = ffg_init(max_limbs);
    if (rc) ff_gpu_failed("init", ffg_last_error());
    size_t L = ffg_ntt_max_L();
    if (L > g_ntt_max_L) g_ntt_max_L = L;
    ffg_set_ntt_max_L(g_ntt_max_L);
}

int ff_max_lg = NTT_MAX_LG; /* lowered by ffg_set_max_lg through ff_set_max_lg */

static int ntt_fits(const Big *a, const Big *b) {
    return 2 * (a->n + b->n) - 1 <= g_ntt_max_L || g_ntt_max_L >= ((size_t)1 << ff_max_lg);
}

/* The run-time NTT_MAX_LG of this surface and of the GPU layer together. */
int ff_set_max_lg(int lg) {
    int rc = ffg_set_max_lg(lg);
    if (rc) return rc;
    ff_max_lg = lg;
    if (g_ntt_max_L > ((size_t)1 << lg)) g_ntt_max_L = (size_t)1 << lg;
    return 0;
}

Big big_mul_ntt(const Big *a, const Big *b) {
    if (big_is_zero(a) || big_is_zero(b)) return big_from_u64(0);
    ffg_set_ntt_max_L(g_ntt_max_L);
    int sq = a == b;
    size_t cap = a->n + b->n;
    uint64_t *d = xmalloc(cap * sizeof(uint64_t));
    size_t n = 0;
    int rc = ffg_mul_host(d, &n, a->d, a->n, b->d, b->n, sq);
    if (rc) ff_gpu_failed("multiply", ffg_last_error());
    return (Big){d, n};
}

static Big karatsuba_combine(Big *z0, Big *z1, Big *z2, size_t half, size_t n) {
    big_sub_at(z1->d, z1->n, z2, 0);
    big_sub_at(z1->d, z1->n, z0, 0);
    z1->n = normalize_len(z1->d, z1->n);
    uint64_t *d = xcalloc(n, sizeof(uint64_t));
    big_add_at(d, n, z0, 0);
    big_add_at(d, n, z1, half);
    big_add_at(d, n, z2, 2 * half);
    big_free(z0);
    big_free(z1);
    big_free(z2);
    return (Big){d, normalize_len(d, n)};
}

Big big_mul(const Big *a, const Big *b) {
    size_t minlen = a->n < b->n ? a->n : b->n;
    if (a == b) return big_sqr(a);
    if (minlen <= KARATSUBA_THRESHOLD_LIMBS) return big_mul_schoolbook(a, b);
    if (minlen >= NTT_THRESHOLD_LIMBS && ntt_fits(a, b)) return big_mul_ntt(a, b);
    if (minlen >= TOOM3_THRESHOLD_LIMBS) return big_mul_toom3(a, b);
    size_t half = (a->n > b->n ? a->n : b->n) / 2;
    Big al = view_slice(a, 0, half), ah = view_slice(a, half, a->n);
    Big bl = view_slice(b, 0, half), bh = view_slice(b, half, b->n);
    Big z0 = big_mul(&al, &bl), z2 = big_mul(&ah, &bh);
    Big sa = big_add(&al, &ah), sb = big_add(&bl, &bh);
    Big z1 = big_mul(&sa, &sb);
    big_free(&sa);
    big_free(&sb);
    return karatsuba_combine(&z0, &z1, &z2, half, a->n + b->n);
}

Big big_sqr(const Big *a) {
    if (a->n <= KARATSUBA_THRESHOLD_LIMBS) return big_sqr_schoolbook(a);
    if (a->n >= NTT_THRESHOLD_LIMBS && ntt_fits(a, a)) return big_mul_ntt(a, a);
    if (a->n >= TOOM3_THRESHOLD_LIMBS) return big_mul_toom3(a, a);
    size_t half = a->n / 2;
    Big al = view_slice(a, 0, half), ah = view_slice(a, half, a->n);
    Big z0 = big_sqr(&al), z2 = big_sqr(&ah);
    Big sa = big_add(&al, &ah);
    Big z1 = big_sqr(&sa);
    big_free(&sa);
    return karatsuba_combine(&z0, &z1, &z2, half, 2 * a->n);
}

/* ------------------------------------------------------------ Toom-3 */

static SBig sb_wrap(Big m, int neg) { return (SBig){big_is_zero(&m) ? 0 : neg, m}; }
static void sb_free(SBig *x) { big_free(&x->mag); }

static SBig sb_add(const SBig *x, const SBig *y) {
    if (x->neg == y->neg) return sb_wrap(big_add(&x->mag, &y->mag), x->neg);
    int c = big_cmp(&x->mag, &y->mag);
    if (c == 0) return sb_wrap(big_from_u64(0), 0);
    return c > 0 ? sb_wrap(big_sub(&x->mag, &y->mag), x->neg) : sb_wrap(big_sub(&y->mag, &x->mag), y->neg);
}

static SBig sb_sub(const SBig *x, const SBig *y) {
    SBig ny = {big_is_zero(&y->mag) ? 0 : !y->neg, y->mag};
    return sb_add(x, &ny);
}

static SBig sb_diff(const Big *x, const Big *y) {
    return big_cmp(x, y) >= 0 ? sb_wrap(big_sub(x, y), 0) : sb_wrap(big_sub(y, x), 1);
}

/* Exact division by 2 or 3 (the interpolation's divisions are exact). */
static SBig sb_div(const SBig *x, uint32_t dv) {
    Big t = big_copy(&x->mag);
    unsigned __int128 rem = 0;
    for (size_t i = t.n; i-- > 0;) {
        unsigned __int128 cur = (rem << 64) | t.d[i];
        t.d[i] = (uint64_t)(cur / dv);
        rem = cur % dv;
    }
    t.n = normalize_len(t.d, t.n);
    return sb_wrap(t, x->neg);
}

static Big t3mul(const Big *x, const Big *y, int sq) { return sq ? big_sqr(x) : big_mul(x, y); }

/* Toom-Cook 3 (src/mul_basic.c:175-252): evaluate at 0, 1, -1, -2, inf,
   five products of a third of the size, interpolate. */
Big big_mul_toom3(const Big *a, const Big *b) {
    int sq = a == b;
    size_t maxlen = a->n > b->n ? a->n : b->n, k = (maxlen + 2) / 3;
    Big x[3] = {view_slice(a, 0, k), view_slice(a, k, 2 * k), view_slice(a, 2 * k, a->n)};
    Big y[3] = {view_slice(b, 0, k), view_slice(b, k, 2 * k), view_slice(b, 2 * k, b->n)};
    Big e1[2];
    SBig em1[2], em2[2];
    for (int s = 0; s < (sq ? 1 : 2); s++) {
        const Big *v = s ? y : x;
        Big t = big_add(&v[0], &v[2]);
        e1[s] = big_add(&t, &v[1]);
        em1[s] = sb_diff(&t, &v[1]);
        big_free(&t);
        Big x24 = big_shl_bits(&v[2], 2), x12 = big_shl_bits(&v[1], 1), s04 = big_add(&v[0], &x24);
        em2[s] = sb_diff(&s04, &x12);
        big_free(&x24);
        big_free(&x12);
        big_free(&s04);
    }
    int o = sq ? 0 : 1;
    Big R0m = t3mul(&x[0], &y[0], sq), Rim = t3mul(&x[2], &y[2], sq), R1m = t3mul(&e1[0], &e1[o], sq);
    SBig Rm1 = sb_wrap(t3mul(&em1[0].mag, &em1[o].mag, sq), em1[0].neg ^ em1[o].neg);
    SBig Rm2 = sb_wrap(t3mul(&em2[0].mag, &em2[o].mag, sq), em2[0].neg ^ em2[o].neg);
    for (int s = 0; s < (sq ? 1 : 2); s++) {
        big_free(&e1[s]);
        sb_free(&em1[s]);
        sb_free(&em2[s]);
    }
    SBig R0 = sb_wrap(R0m, 0), R1 = sb_wrap(R1m, 0), Ri = sb_wrap(Rim, 0);
    /* r3 = (Rm2 - R1)/3, r1 = (R1 - Rm1)/2, r2 = Rm1 - R0,
       r3 = (r2 - r3)/2 + 2 Rinf, r2 = r2 + r1 - Rinf, r1 = r1 - r3 */
    SBig t = sb_sub(&Rm2, &R1), r3 = sb_div(&t, 3);
    sb_free(&t);
    t = sb_sub(&R1, &Rm1);
    SBig r1 = sb_div(&t, 2);
    sb_free(&t);
    SBig r2 = sb_sub(&Rm1, &R0);
    sb_free(&Rm1);
    sb_free(&Rm2);
    sb_free(&R1);
    t = sb_sub(&r2, &r3);
    SBig h = sb_div(&t, 2);
    sb_free(&t);
    sb_free(&r3);
    SBig ri2 = sb_wrap(big_shl_bits(&Ri.mag, 1), 0);
    r3 = sb_add(&h, &ri2);
    sb_free(&h);
    sb_free(&ri2);
    t = sb_add(&r2, &r1);
    sb_free(&r2);
    r2 = sb_sub(&t, &Ri);
    sb_free(&t);
    t = sb_sub(&r1, &r3);
    sb_free(&r1);
    r1 = t;
    size_t n = a->n + b->n;
    uint64_t *d = xcalloc(n, sizeof(uint64_t));
    big_add_at(d, n, &R0.mag, 0);
    big_add_at(d, n, &r1.mag, k);
    big_add_at(d, n, &r2.mag, 2 * k);
    big_add_at(d, n, &r3.mag, 3 * k);
    big_add_at(d, n, &Ri.mag, 4 * k);
    sb_free(&R0);
    sb_free(&r1);
    sb_free(&r2);
    sb_free(&r3);
    sb_free(&Ri);
    return (Big){d, normalize_len(d, n)};
}
