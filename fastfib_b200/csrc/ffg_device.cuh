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
// pad(i) = i + i/32 (ffg_lines.cuh): a forward transform is decimation in
// frequency (natural order in, digit-reversed out), the inverse decimation
// in time (digit-reversed in, natural out), so no permutation pass is ever
// needed.
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
    const uint2 *stw;  // step twiddles ω_N^(j brev_M(s)) (Shoup pairs), one table per (stride, radix)
    const uint2 *istw; // the same with ω_N^-1
    const uint4 *r3f; // r3f[2^n + j] = (ω_R^j, s, ω_R^2j, s) for R = 3 2^n, j < 2^n
    const uint4 *r3i; // the same with ω_R^-1
    const uint32_t *twl; // ω_M^e * 2^32 mod p for e < FFG_TW_LO      (M = 3 2^25)
    const uint32_t *twh; // ω_M^(e FFG_TW_LO) * 2^32 mod p, e < M / FFG_TW_LO
};

struct Primes3 {
    PrimeDev pr[3];
};

// Constants of the in-register line transforms, in constant memory: ω_32^e
// and ω_32^-e (e < 16) as Shoup pairs, the cube roots of unity, and the
// offset of the step twiddle table of (stride 2^sl, radix 2^M) at sl * 6 + M.
struct LineConsts {
    uint2 f[3][16];
    uint2 i[3][16];
    uint2 w3[3], v3[3];
    uint32_t pinv[3];
    uint32_t tw_off[15 * 6];
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

// The step schedule of a 2^n block: radix-16 steps while more than 9 levels
// remain (stride >= 32), then one step down to stride 32, then the last step
// on contiguous groups (stride 1, radix up to 32, no twiddles).  Returns the number of steps; step i has
// radix 2^m[i] and stride 2^sl[i], listed in DIF order (largest stride first).
__host__ __device__ inline int schedule(uint32_t n, int (&m)[4], int (&sl)[4]) {
    int k = 0, s = (int)n;
    while (s > 9) {
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

// Frequency index held at line position pos after a forward line transform.
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
