// Device-side arithmetic and in-shared-memory transforms for the three-prime
// NTT multiply, written for sm_100a (B200).
//
// Primes, as in the reference (src/ntt_arith.c:48-52): p1 = 63*2^25+1 (g=5),
// p2 = 15*2^27+1 (g=31), p3 = 27*2^26+1 (g=13).  Every p < 2^31, so a sum of
// two residues fits in 32 bits and one unsigned min() reduces it.  Residues
// are kept canonical in [0, p) in standard (not Montgomery) form.
//
// Two modular products are used:
//  * Shoup's product by a known constant w with ws = floor(w 2^32 / p):
//    q = umulhi(a, ws), r = a w - q p  in [0, 2p) for any 32-bit a; then one
//    min() -- three integer multiplies.  Every transform twiddle is a table
//    pair (w, ws).
//  * Montgomery's product a b 2^-32 mod p for two variable residues (the
//    pointwise product, and the four-step twiddles ω^(n2 k1) that are built
//    from two small tables in Montgomery form).
//
// Transforms run on "lines" held in shared memory at padded positions
// pad(i) = i + i/32: with that padding every access pattern below (32
// consecutive j of a wide step, or a thread's own 2^M consecutive elements in
// the last step) is free of bank conflicts.  A line of length N = 3^t 2^n is
// transformed by an optional radix-3 step (stride 2^n) followed by radix-2^M
// steps on each 2^n block; each thread keeps one group of 2^M elements in
// registers per step.  The forward transform is decimation in frequency
// (natural order in, digit-reversed out), the inverse decimation in time
// (digit-reversed in, natural out), so no permutation pass is ever needed.
#pragma once
#include <cstdint>

#ifndef FFG_DEV_INLINE
#define FFG_DEV_INLINE __device__ __forceinline__
#endif

namespace ffg {

// One prime's constants and device tables, passed to kernels by value.
struct PrimeDev {
    uint32_t p;       // the prime
    uint32_t pinv;    // p^-1 mod 2^32 (Montgomery)
    uint32_t w3, w3s; // a primitive cube root of unity ω_3 and its Shoup quotient
    uint32_t v3, v3s; // ω_3^-1 and its Shoup quotient
    uint32_t c32, c32s; // 2^32 mod p and its Shoup quotient (digit reduction)
    const uint2 *rt;  // rt[h + i]  = (ω_2h^i,  Shoup) for 1 <= h < 2^FFG_LINE_LG
    const uint2 *irt; // irt[h + i] = (ω_2h^-i, Shoup)
    const uint4 *r3f; // r3f[2^n + j] = (ω_R^j, s, ω_R^2j, s) for R = 3 2^n, j < 2^n
    const uint4 *r3i; // the same with ω_R^-1
    const uint32_t *twl; // ω_M^e * 2^32 mod p for e < FFG_TW_LO      (M = 3 2^25)
    const uint32_t *twh; // ω_M^(e FFG_TW_LO) * 2^32 mod p, e < M / FFG_TW_LO
};

struct Primes3 {
    PrimeDev pr[3];
};

constexpr int FFG_LINE_LG = 14;             // longest power-of-2 line in shared memory
constexpr uint32_t FFG_TW_LO_LG = 12;
constexpr uint32_t FFG_TW_LO = 1u << FFG_TW_LO_LG;
constexpr uint64_t FFG_M = 3ull << 25;      // every supported length divides M

FFG_DEV_INLINE uint32_t pad_idx(uint32_t i) { return i + (i >> 5); }

FFG_DEV_INLINE uint32_t add_mod(uint32_t a, uint32_t b, uint32_t p) {
    uint32_t s = a + b;
    return min(s, s - p);
}
FFG_DEV_INLINE uint32_t sub_mod(uint32_t a, uint32_t b, uint32_t p) {
    uint32_t d = a - b;
    return min(d, d + p);
}
// a w mod p for any 32-bit a; (w, ws) a Shoup pair.
FFG_DEV_INLINE uint32_t shoup(uint32_t a, uint32_t w, uint32_t ws, uint32_t p) {
    uint32_t q = __umulhi(a, ws);
    uint32_t r = a * w - q * p;
    return min(r, r - p);
}
// a b 2^-32 mod p for a, b in [0, p).
FFG_DEV_INLINE uint32_t mont(uint32_t a, uint32_t b, uint32_t p, uint32_t pinv) {
    uint64_t t = (uint64_t)a * b;
    uint32_t m = (uint32_t)t * pinv;
    uint32_t r = (uint32_t)(t >> 32) - __umulhi(m, p);
    return min(r, r + p);
}

// Forward (DIF) butterfly: (x, y) -> (x + y, (x - y) w).
FFG_DEV_INLINE void bf_dif(uint32_t &x, uint32_t &y, uint2 w, uint32_t p) {
    uint32_t s = add_mod(x, y, p);
    y = shoup(x - y + p, w.x, w.y, p);
    x = s;
}
// Inverse (DIT) butterfly: (x, y) -> (x + y w, x - y w).
FFG_DEV_INLINE void bf_dit(uint32_t &x, uint32_t &y, uint2 w, uint32_t p) {
    uint32_t t = shoup(y, w.x, w.y, p);
    y = sub_mod(x, t, p);
    x = add_mod(x, t, p);
}

// M levels of the DIF on one group x[0..2^M) = elements j + t S of a block of
// size 2^M S: level l pairs t and t + 2^(M-1-l) with twiddle
// ω_2h^(j + (t mod 2^(M-1-l)) S), h = S 2^(M-1-l).
template <int M>
FFG_DEV_INLINE void group_dif(uint32_t (&x)[1 << M], const uint2 *__restrict__ rt, uint32_t j, uint32_t S,
                              uint32_t p) {
#pragma unroll
    for (int l = 0; l < M; l++) {
        const int half = 1 << (M - 1 - l);
#pragma unroll
        for (int t = 0; t < (1 << M); t++) {
            if (t & half) continue;
            uint2 w = __ldg(&rt[S * half + j + (t & (half - 1)) * S]);
            bf_dif(x[t], x[t + half], w, p);
        }
    }
}

// M levels of the DIT (the mirror of group_dif): level l pairs t and t + 2^l
// with twiddle ω_2h^-(j + (t mod 2^l) S), h = S 2^l.
template <int M>
FFG_DEV_INLINE void group_dit(uint32_t (&x)[1 << M], const uint2 *__restrict__ irt, uint32_t j, uint32_t S,
                              uint32_t p) {
#pragma unroll
    for (int l = 0; l < M; l++) {
        const int half = 1 << l;
#pragma unroll
        for (int t = 0; t < (1 << M); t++) {
            if (t & half) continue;
            uint2 w = __ldg(&irt[S * half + j + (t & (half - 1)) * S]);
            bf_dit(x[t], x[t + half], w, p);
        }
    }
}

// Shape of the lines a CTA transforms: `lines` lines of length 3^r3 2^n, line
// k at shared offset k * stride (in words, padding included).
struct LineSet {
    uint32_t lines;
    uint32_t n;      // log2 of the power-of-2 part
    uint32_t r3;     // 1: a radix-3 step splits each line into three 2^n blocks
    uint32_t stride; // shared-memory words between consecutive lines
};

// One radix-2^M step (stride S) over every block of every line: the CTA's
// threads share the groups.  dir > 0: DIF, else DIT.
template <int M, bool DIF>
FFG_DEV_INLINE void step_pow2(uint32_t *s, const LineSet &ls, const uint2 *__restrict__ tab, uint32_t S,
                              uint32_t p) {
    const uint32_t per_block = (1u << ls.n) >> M; // groups per 2^n block
    const uint32_t nblk3 = ls.r3 ? 3 : 1;
    const uint32_t total = per_block * nblk3 * ls.lines;
    for (uint32_t g = threadIdx.x; g < total; g += blockDim.x) {
        uint32_t gb = g % per_block, rest = g / per_block;
        uint32_t q = rest % nblk3, line = rest / nblk3;
        uint32_t sb = gb / S, j = gb % S;
        uint32_t base = (q << ls.n) + (sb << M) * S + j;
        uint32_t *L = s + line * ls.stride;
        uint32_t x[1 << M];
#pragma unroll
        for (int t = 0; t < (1 << M); t++) x[t] = L[pad_idx(base + t * S)];
        if (DIF) group_dif<M>(x, tab, j, S, p);
        else group_dit<M>(x, tab, j, S, p);
#pragma unroll
        for (int t = 0; t < (1 << M); t++) L[pad_idx(base + t * S)] = x[t];
    }
}

// The step schedule of a 2^n block: radix-16 steps while more than 10 levels
// remain (stride >= 64), then one step down to stride 32, then the last step
// on contiguous groups (stride 1).  Returns the number of steps; step i has
// radix 2^m[i] and stride 2^sl[i], listed in DIF order (largest stride first).
FFG_DEV_INLINE int schedule(uint32_t n, int (&m)[4], int (&sl)[4]) {
    int k = 0, s = (int)n;
    while (s > 10) {
        m[k] = 4;
        sl[k] = s - 4;
        s -= 4;
        k++;
    }
    if (s > 5) {
        m[k] = s - 5;
        sl[k] = 5;
        s = 5;
        k++;
    }
    m[k] = s;
    sl[k] = 0;
    return k + 1;
}

template <bool DIF>
FFG_DEV_INLINE void step_dispatch(int m, uint32_t *s, const LineSet &ls, const uint2 *tab, uint32_t S, uint32_t p) {
    switch (m) {
    case 1: step_pow2<1, DIF>(s, ls, tab, S, p); break;
    case 2: step_pow2<2, DIF>(s, ls, tab, S, p); break;
    case 3: step_pow2<3, DIF>(s, ls, tab, S, p); break;
    case 4: step_pow2<4, DIF>(s, ls, tab, S, p); break;
    case 5: step_pow2<5, DIF>(s, ls, tab, S, p); break;
    default: break;
    }
}

// Radix-3 DIF step on every line: x_q at j + q 2^n (q = 0, 1, 2) ->
//   y0 = x0 + x1 + x2
//   y1 = (x0 - x2 + ω3 (x1 - x2)) ω_R^j
//   y2 = (x0 - x1 - ω3 (x1 - x2)) ω_R^2j          (ω3^2 = -1 - ω3)
FFG_DEV_INLINE void step_r3_dif(uint32_t *s, const LineSet &ls, const PrimeDev &P) {
    const uint32_t B = 1u << ls.n, total = B * ls.lines, p = P.p;
    for (uint32_t g = threadIdx.x; g < total; g += blockDim.x) {
        uint32_t j = g % B, line = g / B;
        uint32_t *L = s + line * ls.stride;
        uint32_t x0 = L[pad_idx(j)], x1 = L[pad_idx(j + B)], x2 = L[pad_idx(j + 2 * B)];
        uint4 t = __ldg(&P.r3f[B + j]);
        uint32_t u = shoup(x1 - x2 + p, P.w3, P.w3s, p);
        uint32_t y0 = add_mod(add_mod(x0, x1, p), x2, p);
        uint32_t v1 = add_mod(sub_mod(x0, x2, p), u, p);
        uint32_t v2 = sub_mod(sub_mod(x0, x1, p), u, p);
        L[pad_idx(j)] = y0;
        L[pad_idx(j + B)] = shoup(v1, t.x, t.y, p);
        L[pad_idx(j + 2 * B)] = shoup(v2, t.z, t.w, p);
    }
}

// Radix-3 DIT step (inverse of step_r3_dif up to the factor 3): with
// z1 = y1 ω_R^-j, z2 = y2 ω_R^-2j and ν = ω3^-1,
//   x0 = y0 + z1 + z2,  x1 = y0 - z2 + ν (z1 - z2),  x2 = y0 - z1 - ν (z1 - z2).
FFG_DEV_INLINE void step_r3_dit(uint32_t *s, const LineSet &ls, const PrimeDev &P) {
    const uint32_t B = 1u << ls.n, total = B * ls.lines, p = P.p;
    for (uint32_t g = threadIdx.x; g < total; g += blockDim.x) {
        uint32_t j = g % B, line = g / B;
        uint32_t *L = s + line * ls.stride;
        uint4 t = __ldg(&P.r3i[B + j]);
        uint32_t y0 = L[pad_idx(j)];
        uint32_t z1 = shoup(L[pad_idx(j + B)], t.x, t.y, p);
        uint32_t z2 = shoup(L[pad_idx(j + 2 * B)], t.z, t.w, p);
        uint32_t u = shoup(z1 - z2 + p, P.v3, P.v3s, p);
        L[pad_idx(j)] = add_mod(add_mod(y0, z1, p), z2, p);
        L[pad_idx(j + B)] = add_mod(sub_mod(y0, z2, p), u, p);
        L[pad_idx(j + 2 * B)] = sub_mod(sub_mod(y0, z1, p), u, p);
    }
}

// Forward transform of every line in shared memory (natural order in,
// digit-reversed out: position q 2^n + i holds frequency q + 3 brev_n(i), or
// brev_n(i) without the radix-3 step).
FFG_DEV_INLINE void lines_forward(uint32_t *s, const LineSet &ls, const PrimeDev &P) {
    if (ls.r3) {
        step_r3_dif(s, ls, P);
        __syncthreads();
    }
    int m[4], sl[4];
    int k = schedule(ls.n, m, sl);
    for (int i = 0; i < k; i++) {
        step_dispatch<true>(m[i], s, ls, P.rt, 1u << sl[i], P.p);
        __syncthreads();
    }
}

// Inverse transform (digit-reversed in, natural out), unnormalized: the
// result is N times the inverse DFT.
FFG_DEV_INLINE void lines_inverse(uint32_t *s, const LineSet &ls, const PrimeDev &P) {
    int m[4], sl[4];
    int k = schedule(ls.n, m, sl);
    for (int i = k - 1; i >= 0; i--) {
        step_dispatch<false>(m[i], s, ls, P.irt, 1u << sl[i], P.p);
        __syncthreads();
    }
    if (ls.r3) {
        step_r3_dit(s, ls, P);
        __syncthreads();
    }
}

// Frequency index held at line position pos after lines_forward.
FFG_DEV_INLINE uint32_t freq_of(uint32_t pos, uint32_t n, uint32_t r3) {
    uint32_t i = pos & ((1u << n) - 1);
    uint32_t rev = n ? (__brev(i) >> (32 - n)) : 0;
    return r3 ? (pos >> n) + 3 * rev : rev;
}

// ω_L^e (e < L, L | M) in Montgomery form, from the two small tables:
// ω_M^E with E = e M / L = Eh 2^12 + El.
FFG_DEV_INLINE uint32_t tw_mont(const PrimeDev &P, uint64_t E) {
    uint32_t lo = __ldg(&P.twl[E & (FFG_TW_LO - 1)]);
    uint32_t hi = __ldg(&P.twh[E >> FFG_TW_LO_LG]);
    return mont(lo, hi, P.p, P.pinv); // (ω^El 2^32)(ω^Eh 2^32) 2^-32
}

// b-bit digit i of the limb array a (na limbs), zero past the end: the
// reference's Src reader (src/ntt_kernels.c:29-74).
FFG_DEV_INLINE uint64_t digit_at(const uint64_t *__restrict__ a, uint64_t na, uint64_t i, uint32_t b) {
    uint64_t bit = i * b, q = bit >> 6;
    uint32_t off = (uint32_t)(bit & 63);
    if (q >= na) return 0;
    uint64_t lo = __ldg(&a[q]);
    uint64_t hi = (off + b > 64 && q + 1 < na) ? __ldg(&a[q + 1]) : 0;
    uint64_t v = off ? (lo >> off) | (hi << (64 - off)) : lo;
    return v & ((1ull << b) - 1);
}

// A digit v < 2^35 reduced mod p: v = h 2^32 + l with h < 8, so
// v mod p = (l mod p) + h (2^32 mod p); l < 2^32 < 3p needs two conditional
// subtractions and the high part one Shoup product.
FFG_DEV_INLINE uint32_t reduce_digit(uint64_t v, const PrimeDev &P) {
    uint32_t l = (uint32_t)v, h = (uint32_t)(v >> 32), p = P.p;
    l = min(l, l - p);
    l = min(l, l - p);
    return add_mod(l, shoup(h, P.c32, P.c32s, p), p);
}

} // namespace ffg
