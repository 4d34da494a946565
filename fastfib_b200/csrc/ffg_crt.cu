// CRT recombination and the fast-doubling linear passes, for sm_100a.
//
// k_crt: one CTA per 2048 coefficients (= 32 * width output limbs exactly).
//   1. Garner's method per coefficient (the reference's crt_garner8,
//      src/crt.c:38-64), in parallel, for the block plus a halo of the few
//      coefficients below it that reach into its limbs:
//        x2 = (r2 - r1) p1^-1 mod p2,  x3 = ((r3 - r1) p1^-1 - x2) p2^-1 mod p3,
//        X  = r1 + x2 p1 + x3 p1 p2  < p1 p2 p3 < 2^93.
//   2. Every limb j sums the slices of the coefficients X_i 2^(i b) that
//      overlap it (3-6 of them): the column sum lo_j + 2^64 hi_j.  This is the
//      reference's crt_pack64 (src/crt.c:70-87) with the running carry turned
//      into per-limb sums.
//   3. cta_resolve (ffg_ripple.cuh) settles the one-bit ripples; the CTA
//      that finishes last settles the carries between CTAs (settle_cta).
// A small signed constant is added to the product on the way (the final
// +-2 of fast doubling, src/fib.c:249) in two's complement over the output.
//
// k_lin: out = alpha s1 + beta s2 + gamma over len limbs, two outputs per
// launch (the reference's step_proc / last_proc, src/fib.c:37-62, 123-143);
// negative terms in two's complement (-s = ~s + 1 mod 2^(64 len)), so every
// column sum is non-negative and the same ripple settle applies.
#include <cstdlib>

#include "ffg_internal.h"
#include "ffg_ripple.cuh"

namespace ffg {

typedef unsigned __int128 u128;

constexpr uint32_t CRT_COEF = 2048;     // coefficients per CTA
constexpr uint32_t CRT_THREADS = 256;
constexpr uint32_t CRT_HALO_MAX = 24;   // ceil(156 / b) + 1 for b >= 8, rounded up to 4
constexpr uint32_t CRT_NL_MAX = 32 * 35;
constexpr uint32_t CRT_NL_PER_W = 32;   // limbs per CTA = 32 * width

FFG_DEV_INLINE int64_t floor_div(int64_t a, int64_t b) { return a >= 0 ? a / b : -((-a + b - 1) / b); }
FFG_DEV_INLINE int32_t floor_div32(int32_t a, int32_t b) { return a >= 0 ? a / b : -((-a + b - 1) / b); }

FFG_DEV_INLINE uint32_t crt_ctas_dev(uint64_t nlimbs, uint32_t width) {
    const uint64_t NL = (uint64_t)CRT_NL_PER_W * width;
    return (uint32_t)((nlimbs + NL - 1) / NL);
}

FFG_DEV_INLINE void crt_block(const GarnerConst &K, const CrtJob &J, uint32_t cta);

__global__ void __launch_bounds__(CRT_THREADS) k_crt(GarnerConst K, CrtJob J) { crt_block(K, J, blockIdx.x); }

// Up to two CRTs by value (the doubling step's two squarings): product
// blockIdx.y, its CTA blockIdx.x.
struct CrtPair {
    CrtJob j[2];
};
__global__ void __launch_bounds__(CRT_THREADS) k_crt_pair(GarnerConst K, CrtPair P) {
    const CrtJob &J = P.j[blockIdx.y];
    if (blockIdx.x >= crt_ctas_dev(J.nlimbs, J.width)) return;
    crt_block(K, J, blockIdx.x);
}

// A batch of CRTs: product blockIdx.y, its CTA blockIdx.x (CTAs past the
// product's own count return at once, all threads together).
__global__ void __launch_bounds__(CRT_THREADS) k_crt_batch(GarnerConst K, const CrtJob *__restrict__ jobs) {
    const CrtJob J = jobs[blockIdx.y];
    if (blockIdx.x >= crt_ctas_dev(J.nlimbs, J.width)) return;
    crt_block(K, J, blockIdx.x);
}

// CRTs of any sizes in one launch: CTA b runs CTA b - first[j] of job j,
// first[j] <= b < first[j + 1] (first: count + 1 prefix sums of the jobs'
// CTA counts), found by binary search.
__global__ void __launch_bounds__(CRT_THREADS) k_crt_flat(GarnerConst K, const CrtJob *__restrict__ jobs,
                                                         const uint32_t *__restrict__ first, uint32_t count) {
    const uint32_t b = blockIdx.x;
    uint32_t lo = 0, hi = count; // invariant: first[lo] <= b < first[hi]
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) / 2;
        if (__ldg(&first[mid]) <= b) lo = mid;
        else hi = mid;
    }
    const CrtJob J = jobs[lo];
    crt_block(K, J, b - __ldg(&first[lo]));
}

// Garner's recombination of one coefficient's residues: X < p1 p2 p3 < 2^93.
FFG_DEV_INLINE u128 garner(const GarnerConst &K, uint32_t r1, uint32_t r2, uint32_t r3) {
    const uint32_t p1 = K.p[0], p2 = K.p[1], p3 = K.p[2];
    const uint32_t x1m2 = min(r1, r1 - p2);
    const uint32_t x2 = shoup(r2 - x1m2 + p2, K.i12, K.i12s, p2);
    const uint32_t x1m3 = min(r1, r1 - p3);
    const uint32_t t3 = shoup(r3 - x1m3 + p3, K.i13, K.i13s, p3);
    const uint32_t x2m3 = min(x2, x2 - p3);
    const uint32_t x3 = shoup(t3 - x2m3 + p3, K.i23, K.i23s, p3);
    return (u128)((uint64_t)x2 * p1 + r1) + (u128)x3 * K.p12;
}

// Column sum lo + 2^64 hi of limb j (relative to the CTA's first limb) over
// the values Z_i 2^(i b) (i relative to the CTA's first coefficient, stored
// from -halo), every Z_i below 2^(top + 1).  B: the width when known at
// compile time (0: bw at run time); indices and shifts fit 32 bits (j is at
// most 32 * 35 limbs, i at most 2048 + halo coefficients).
template <int B>
FFG_DEV_INLINE void column_sum_w(const uint64_t *Zlo, const uint32_t *Zhi, int32_t j, uint32_t bw, int32_t halo,
                                 int32_t top, uint64_t &s_lo, uint32_t &s_hi) {
    const int32_t b = B ? B : (int32_t)bw;
    const int32_t ilo = floor_div32(64 * j - top + b - 1, b), ihi = floor_div32(64 * j + 63, b);
    s_lo = 0;
    s_hi = 0;
    for (int32_t i = ilo < -halo ? -halo : ilo; i <= ihi; i++) {
        const u128 X = ((u128)Zhi[i + halo] << 64) | Zlo[i + halo];
        const int32_t sft = i * b - 64 * j;
        const uint64_t part = sft >= 0 ? (uint64_t)(X << sft) : (uint64_t)(X >> (-sft));
        s_lo += part;
        s_hi += s_lo < part;
    }
}

// The same with big_mul_ntt's widths (32..35) as compile-time divisors; b is
// the same for every thread of a CTA, so the switch does not diverge.
FFG_DEV_INLINE void column_sum(const uint64_t *Zlo, const uint32_t *Zhi, int32_t j, uint32_t b, int32_t halo,
                               int32_t top, uint64_t &s_lo, uint32_t &s_hi) {
    switch (b) {
    case 32: column_sum_w<32>(Zlo, Zhi, j, b, halo, top, s_lo, s_hi); return;
    case 33: column_sum_w<33>(Zlo, Zhi, j, b, halo, top, s_lo, s_hi); return;
    case 34: column_sum_w<34>(Zlo, Zhi, j, b, halo, top, s_lo, s_hi); return;
    case 35: column_sum_w<35>(Zlo, Zhi, j, b, halo, top, s_lo, s_hi); return;
    default: column_sum_w<0>(Zlo, Zhi, j, b, halo, top, s_lo, s_hi); return;
    }
}

FFG_DEV_INLINE void crt_block(const GarnerConst &K, const CrtJob &J, uint32_t cta) {
    extern __shared__ __align__(16) unsigned char sm[];
    uint64_t *Xlo = (uint64_t *)sm;                              // CRT_COEF + halo
    uint64_t *lo = Xlo + CRT_COEF + CRT_HALO_MAX;                // NL limbs
    uint32_t *Xhi = (uint32_t *)(lo + CRT_NL_MAX);               // CRT_COEF + halo
    uint32_t *hi = Xhi + CRT_COEF + CRT_HALO_MAX;                // NL
    uint32_t *gG = hi + CRT_NL_MAX, *gP = gG + CRT_NL_MAX / 32, *gin = gP + CRT_NL_MAX / 32;
    __shared__ uint32_t hiprev_s;

    const uint32_t b = J.width, NL = CRT_NL_PER_W * b;
    const int32_t halo = (int32_t)(((156 + b - 1) / b + 1 + 3) & ~3u);
    const int64_t ibase = (int64_t)cta * CRT_COEF;

    // residues in 16-byte vectors of 4 coefficients, every load of the thread
    // issued before any arithmetic (ibase - halo and the strides are multiples
    // of 4, and every residue array is a multiple of 16 words long)
    constexpr int VPT = (CRT_COEF + CRT_HALO_MAX) / 4 / CRT_THREADS + 1; // vectors per thread
    const int32_t nvec = ((int32_t)CRT_COEF + halo) / 4;
    uint4 rv[VPT][3];
#pragma unroll
    for (int v = 0; v < VPT; v++) {
        const int32_t t4 = (int32_t)threadIdx.x + v * (int32_t)blockDim.x;
        const int64_t gi = ibase - halo + 4 * (int64_t)t4;
        const bool in = t4 < nvec && gi >= 0 && (uint64_t)gi < J.conv;
#pragma unroll
        for (int k = 0; k < 3; k++)
            rv[v][k] = in ? __ldg((const uint4 *)(J.y + k * J.y_stride + gi)) : make_uint4(0, 0, 0, 0);
    }
#pragma unroll
    for (int v = 0; v < VPT; v++) {
        const int32_t t4 = (int32_t)threadIdx.x + v * (int32_t)blockDim.x;
        if (t4 >= nvec) break;
        const int64_t gi0 = ibase - halo + 4 * (int64_t)t4;
        const uint32_t r1s[4] = {rv[v][0].x, rv[v][0].y, rv[v][0].z, rv[v][0].w};
        const uint32_t r2s[4] = {rv[v][1].x, rv[v][1].y, rv[v][1].z, rv[v][1].w};
        const uint32_t r3s[4] = {rv[v][2].x, rv[v][2].y, rv[v][2].z, rv[v][2].w};
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const int64_t gi = gi0 + e;
            const u128 X = gi >= 0 && (uint64_t)gi < J.conv ? garner(K, r1s[e], r2s[e], r3s[e]) : (u128)0;
            Xlo[4 * t4 + e] = (uint64_t)X;
            Xhi[4 * t4 + e] = (uint32_t)(X >> 64);
        }
    }
    __syncthreads();

    // column sums; j = -1 (the limb below the CTA) only for its high part
    const uint64_t j0 = (uint64_t)cta * NL;
    const bool neg_add = J.add < 0;
    for (int32_t j = (int32_t)threadIdx.x - 1; j < (int32_t)NL; j += blockDim.x) {
        uint64_t s_lo;
        uint32_t s_hi;
        column_sum(Xlo, Xhi, j, b, halo, 92, s_lo, s_hi);
        // the constant: +add at limb 0, or 2^(64 nlimbs) + add when negative
        const int64_t jabs = (int64_t)j0 + j;
        if (J.add != 0 && jabs >= 0 && (uint64_t)jabs < J.nlimbs) {
            const uint64_t c = jabs == 0 ? (uint64_t)J.add : (neg_add ? ~0ull : 0ull);
            s_lo += c;
            s_hi += s_lo < c;
        }
        if (j < 0) hiprev_s = s_hi;
        else {
            lo[j] = s_lo;
            hi[j] = s_hi;
        }
    }
    __syncthreads();
    const uint32_t map = cta_resolve(lo, hi, cta ? hiprev_s : 0, NL, gG, gP, gin);
    for (uint32_t j = threadIdx.x; j < NL && j0 + j < J.nlimbs; j += blockDim.x) J.out[j0 + j] = lo[j];
    if (threadIdx.x == 0) J.maps[cta] = map;
    const uint32_t ncta = crt_ctas_dev(J.nlimbs, b);
    if (ncta > 1 && last_cta(J.ticket, ncta)) {
        settle_cta(J.out, J.nlimbs, NL, J.maps, ncta);
        if (threadIdx.x == 0) *J.ticket = 0;
    }
}

uint32_t crt_ctas(uint64_t nlimbs, uint32_t width) {
    const uint64_t NL = (uint64_t)CRT_NL_PER_W * width;
    return (uint32_t)((nlimbs + NL - 1) / NL);
}

static size_t crt_smem() {
    return (CRT_COEF + CRT_HALO_MAX) * (8 + 4) + CRT_NL_MAX * (8 + 4) + 3 * (CRT_NL_MAX / 32) * 4;
}

static bool g_crt_configured = false;

cudaError_t crt_kernel_load() {
    if (g_crt_configured) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(k_crt, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)crt_smem());
    if (e) return e;
    g_crt_configured = true;
    return cudaSuccess;
}

cudaError_t launch_crt(const Primes3 &P3, const CrtJob &J, cudaStream_t st) {
    (void)P3;
    cudaError_t e0 = crt_kernel_load();
    if (e0) return e0;
    const uint32_t ncta = crt_ctas(J.nlimbs, J.width);
    prof_begin(PK_CRT, st);
    k_crt<<<ncta, CRT_THREADS, crt_smem(), st>>>(garner_const(), J);
    prof_end(PK_CRT, st, 12.0 * (double)J.conv + 8.0 * (double)J.nlimbs);
    return cudaGetLastError();
}

cudaError_t launch_crt_pair(const CrtJob *jobs, uint32_t count, cudaStream_t st) {
    static bool configured = false;
    if (!configured) {
        cudaError_t e = cudaFuncSetAttribute(k_crt_pair, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)crt_smem());
        if (e) return e;
        configured = true;
    }
    if (count == 1) return launch_crt(Primes3{}, jobs[0], st);
    CrtPair P;
    P.j[0] = jobs[0];
    P.j[1] = jobs[1];
    const uint32_t n0 = crt_ctas(jobs[0].nlimbs, jobs[0].width), n1 = crt_ctas(jobs[1].nlimbs, jobs[1].width);
    double bytes = 0;
    for (int i = 0; i < 2; i++) bytes += 12.0 * (double)jobs[i].conv + 8.0 * (double)jobs[i].nlimbs;
    prof_begin(PK_CRT, st);
    k_crt_pair<<<dim3(n0 > n1 ? n0 : n1, 2), CRT_THREADS, crt_smem(), st>>>(garner_const(), P);
    prof_end(PK_CRT, st, bytes);
    return cudaGetLastError();
}

cudaError_t launch_crt_batch(const CrtJob *d_jobs, uint32_t count, uint32_t max_ctas, cudaStream_t st,
                             double bytes) {
    static bool configured = false;
    if (!configured) {
        cudaError_t e =
            cudaFuncSetAttribute(k_crt_batch, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)crt_smem());
        if (e) return e;
        configured = true;
    }
    if (!count) return cudaSuccess;
    prof_begin(PK_CRT, st);
    k_crt_batch<<<dim3(max_ctas, count), CRT_THREADS, crt_smem(), st>>>(garner_const(), d_jobs);
    prof_end(PK_CRT, st, bytes);
    return cudaGetLastError();
}

cudaError_t launch_crt_flat(const CrtJob *d_jobs, const uint32_t *d_first, uint32_t count, uint32_t total_ctas,
                            cudaStream_t st, double bytes) {
    static bool configured = false;
    if (!configured) {
        cudaError_t e = cudaFuncSetAttribute(k_crt_flat, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)crt_smem());
        if (e) return e;
        configured = true;
    }
    if (!count || !total_ctas) return cudaSuccess;
    prof_begin(PK_CRT, st);
    k_crt_flat<<<total_ctas, CRT_THREADS, crt_smem(), st>>>(garner_const(), d_jobs, d_first, count);
    prof_end(PK_CRT, st, bytes);
    return cudaGetLastError();
}

// ------------------------------------------------------ CRT + linear pass
//
// k_crt_lin: the CRT of a doubling step's two squarings and the step's
// linear pass in one launch.  With X1_i, X2_i the coefficients of s1 and s2,
// output k is sum_i (alpha_k X1_i + beta_k X2_i) 2^(i b) + gamma_k.  beta_k
// may be negative; every coefficient gets the bias B = K (2^b - 1), K =
// 2^(94 - b), so that Z_i = alpha_k X1_i + beta_k X2_i + B >= 0 (|beta_k| X2_i
// <= 2 p1 p2 p3 < 2^94 - K) and Z_i < 4 2^93 + 2^94 < 2^96.  Over the N
// coefficients the CTAs cover, sum_i B 2^(i b) = K 2^(N b) - K: adding the
// constant gamma_k + K leaves the output plus K 2^(N b), a multiple of
// 2^(64 len) that falls off the top (N b >= 64 len).  A CTA recombines both
// squarings' residues of its coefficients and writes one output (short
// products: twice the CTAs, gridDim.y = 2) or both in turn (long products,
// where recombining twice costs more than it hides).  The rest is crt_block
// with values of up to 96 bits, and the CTA that finishes last settles both
// outputs' carries.

// Z_k of one coefficient gi from its residues in both squarings.
FFG_DEV_INLINE u128 crt_lin_z(const GarnerConst &K, const CrtLinJob &J, uint32_t k, int64_t gi, u128 X1, u128 X2,
                              u128 bias) {
    if (gi < 0) return 0;
    const uint64_t alpha = (uint64_t)(k ? J.alpha[1] : J.alpha[0]);
    const int64_t beta = k ? J.beta[1] : J.beta[0];
    // alpha > 0; beta of either sign, the sum taken mod 2^128 (exact: 0 <= Z < 2^96)
    const u128 Z = X1 * alpha + bias;
    return beta >= 0 ? Z + X2 * (uint64_t)beta : Z - X2 * (uint64_t)(-beta);
}

// kSplit: output blockIdx.y only, every load of the thread issued first
// (short products: twice the CTAs); else both outputs from one
// recombination, loads vector by vector (fewer registers, more CTAs per SM).
template <bool kSplit>
__global__ void __launch_bounds__(CRT_THREADS) k_crt_lin(GarnerConst K, CrtLinJob J) {
    extern __shared__ __align__(16) unsigned char sm[];
    constexpr uint32_t ZN = CRT_COEF + CRT_HALO_MAX, NZ = kSplit ? 1 : 2;
    uint64_t *Zlo0 = (uint64_t *)sm;                  // NZ x ZN
    uint64_t *lo = Zlo0 + NZ * ZN;                    // NL limbs
    uint32_t *Zhi0 = (uint32_t *)(lo + CRT_NL_MAX);   // NZ x ZN
    uint32_t *hi = Zhi0 + NZ * ZN;                    // NL
    uint32_t *gG = hi + CRT_NL_MAX, *gP = gG + CRT_NL_MAX / 32, *gin = gP + CRT_NL_MAX / 32;
    __shared__ uint32_t hiprev_s;

    const uint32_t kb = kSplit ? blockIdx.y : 0, ke = kSplit ? blockIdx.y + 1 : 2;
    const uint32_t b = J.width, NL = CRT_NL_PER_W * b, cta = blockIdx.x;
    const int32_t halo = (int32_t)(((159 + b - 1) / b + 1 + 3) & ~3u);
    const int64_t ibase = (int64_t)cta * CRT_COEF;
    const u128 bias = ((u128)1 << (94 - b)) * (((u128)1 << b) - 1);

    constexpr int VPT = (CRT_COEF + CRT_HALO_MAX) / 4 / CRT_THREADS + 1;
    constexpr int VPF = kSplit ? VPT : 1; // vectors whose loads are in flight together
    const int32_t nvec = ((int32_t)CRT_COEF + halo) / 4;
#pragma unroll
    for (int v0 = 0; v0 < VPT; v0 += VPF) {
        uint4 rv[VPF][2][3];
#pragma unroll
        for (int v = 0; v < VPF; v++) {
            const int32_t t4 = (int32_t)threadIdx.x + (v0 + v) * (int32_t)blockDim.x;
            const int64_t gi = ibase - halo + 4 * (int64_t)t4;
#pragma unroll
            for (int q = 0; q < 2; q++) {
                const bool in = t4 < nvec && gi >= 0 && (uint64_t)gi < J.conv[q];
#pragma unroll
                for (int c = 0; c < 3; c++)
                    rv[v][q][c] = in ? __ldg((const uint4 *)(J.y[q] + c * J.y_stride + gi)) : make_uint4(0, 0, 0, 0);
            }
        }
#pragma unroll
        for (int v = 0; v < VPF; v++) {
            const int32_t t4 = (int32_t)threadIdx.x + (v0 + v) * (int32_t)blockDim.x;
            if (t4 >= nvec) break;
            const int64_t gi0 = ibase - halo + 4 * (int64_t)t4;
            const uint32_t r[2][3][4] = {{{rv[v][0][0].x, rv[v][0][0].y, rv[v][0][0].z, rv[v][0][0].w},
                                          {rv[v][0][1].x, rv[v][0][1].y, rv[v][0][1].z, rv[v][0][1].w},
                                          {rv[v][0][2].x, rv[v][0][2].y, rv[v][0][2].z, rv[v][0][2].w}},
                                         {{rv[v][1][0].x, rv[v][1][0].y, rv[v][1][0].z, rv[v][1][0].w},
                                          {rv[v][1][1].x, rv[v][1][1].y, rv[v][1][1].z, rv[v][1][1].w},
                                          {rv[v][1][2].x, rv[v][1][2].y, rv[v][1][2].z, rv[v][1][2].w}}};
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const int64_t gi = gi0 + e;
                u128 X1 = 0, X2 = 0;
                if (gi >= 0) {
                    X1 = (uint64_t)gi < J.conv[0] ? garner(K, r[0][0][e], r[0][1][e], r[0][2][e]) : (u128)0;
                    X2 = (uint64_t)gi < J.conv[1] ? garner(K, r[1][0][e], r[1][1][e], r[1][2][e]) : (u128)0;
                }
#pragma unroll
                for (uint32_t z = 0; z < NZ; z++) {
                    const u128 Z = crt_lin_z(K, J, kb + z, gi, X1, X2, bias);
                    Zlo0[z * ZN + 4 * t4 + e] = (uint64_t)Z;
                    Zhi0[z * ZN + 4 * t4 + e] = (uint32_t)(Z >> 64);
                }
            }
        }
    }
    __syncthreads();

    const uint64_t j0 = (uint64_t)cta * NL;
    const uint32_t ncta = gridDim.x;
    for (uint32_t k = kb; k < ke; k++) {
        const uint32_t z = k - kb;
        const uint64_t add = (uint64_t)(k ? J.gamma[1] : J.gamma[0]) + ((uint64_t)1 << (94 - b)); // gamma + K > 0
        for (int32_t j = (int32_t)threadIdx.x - 1; j < (int32_t)NL; j += blockDim.x) {
            uint64_t s_lo;
            uint32_t s_hi;
            column_sum(Zlo0 + z * ZN, Zhi0 + z * ZN, j, b, halo, 95, s_lo, s_hi);
            if (cta == 0 && j == 0) {
                s_lo += add;
                s_hi += s_lo < add;
            }
            if (j < 0) hiprev_s = s_hi;
            else {
                lo[j] = s_lo;
                hi[j] = s_hi;
            }
        }
        __syncthreads();
        const uint32_t map = cta_resolve(lo, hi, cta ? hiprev_s : 0, NL, gG, gP, gin);
        uint64_t *out = k ? J.out[1] : J.out[0];
        for (uint32_t j = threadIdx.x; j < NL && j0 + j < J.len; j += blockDim.x) out[j0 + j] = lo[j];
        if (threadIdx.x == 0) J.maps[(size_t)k * ncta + cta] = map;
        __syncthreads();
    }
    if (ncta > 1 && last_cta(J.ticket, ncta * gridDim.y)) {
        for (int q = 0; q < 2; q++) settle_cta(q ? J.out[1] : J.out[0], J.len, NL, J.maps + (size_t)q * ncta, ncta);
        if (threadIdx.x == 0) *J.ticket = 0;
    }
}

static size_t crt_lin_smem(bool split) {
    return (split ? 1 : 2) * (CRT_COEF + CRT_HALO_MAX) * (8 + 4) + CRT_NL_MAX * (8 + 4) + 3 * (CRT_NL_MAX / 32) * 4;
}

// Products of up to this many CTAs per output run one output per CTA
// (measured on the F(10^8) and F(10^9) chains).
static uint32_t crt_lin_split_max() {
    static long v = -1;
    if (v < 0) {
        const char *e = getenv("FFG_CRT_LIN_SPLIT");
        v = e && *e ? strtol(e, nullptr, 10) : 128;
        if (v < 0) v = 0;
    }
    return (uint32_t)v;
}

cudaError_t launch_crt_lin(const CrtLinJob &J, cudaStream_t st) {
    static bool configured = false;
    if (!configured) {
        cudaError_t e = cudaFuncSetAttribute(k_crt_lin<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)crt_lin_smem(true));
        if (!e)
            e = cudaFuncSetAttribute(k_crt_lin<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)crt_lin_smem(false));
        if (e) return e;
        configured = true;
    }
    if (J.width < 32 || J.width > 35 || J.alpha[0] <= 0 || J.alpha[1] <= 0) return cudaErrorInvalidValue;
    const uint32_t ncta = crt_ctas(J.len, J.width);
    const bool split = ncta <= crt_lin_split_max();
    prof_begin(PK_CRT, st);
    if (split) k_crt_lin<true><<<dim3(ncta, 2), CRT_THREADS, crt_lin_smem(true), st>>>(garner_const(), J);
    else k_crt_lin<false><<<dim3(ncta, 1), CRT_THREADS, crt_lin_smem(false), st>>>(garner_const(), J);
    prof_end(PK_CRT, st, 12.0 * (double)(J.conv[0] + J.conv[1]) + 16.0 * (double)J.len);
    return cudaGetLastError();
}

// ----------------------------------------------------------- schoolbook

// k_school: a batch of schoolbook products (blockIdx.y the product), 256
// threads per CTA and SCHOOL_NL output limbs (columns) per CTA.  Column j
// sums a_i b_(j-i) over the shorter operand into 192 bits (t0, t1, t2); then
// v_j = t0_j + t1_(j-1) + t2_(j-2) < 3 2^64 leaves single-bit ripples for
// cta_resolve, and the last CTA settles the carries between CTAs.
constexpr uint32_t SCHOOL_NL = 1024;
constexpr uint32_t SCHOOL_THREADS = 256;

__host__ __device__ uint32_t school_ctas(uint64_t nlimbs) { return (uint32_t)((nlimbs + SCHOOL_NL - 1) / SCHOOL_NL); }

FFG_DEV_INLINE void school_col(const SchoolJob &J, int64_t j, uint64_t &t0, uint64_t &t1, uint64_t &t2) {
    t0 = t1 = t2 = 0;
    if (j < 0 || (uint64_t)j >= J.na + J.nb - 1) return;
    // iterate over the shorter operand
    const bool a_short = J.na <= J.nb;
    const uint64_t *S = a_short ? J.a : J.b, *Lg = a_short ? J.b : J.a;
    const int64_t ns = (int64_t)(a_short ? J.na : J.nb), nl = (int64_t)(a_short ? J.nb : J.na);
    const int64_t i0 = j - nl + 1 > 0 ? j - nl + 1 : 0, i1 = j < ns - 1 ? j : ns - 1;
    for (int64_t i = i0; i <= i1; i++) {
        const u128 pr = (u128)__ldg(&S[i]) * __ldg(&Lg[j - i]);
        const uint64_t lo = (uint64_t)pr, hi = (uint64_t)(pr >> 64);
        t0 += lo;
        const uint64_t c0 = t0 < lo;
        const uint64_t h = hi + c0; // hi < 2^64 - 1, so no wrap
        t1 += h;
        t2 += t1 < h;
    }
}

FFG_DEV_INLINE void school_block(const SchoolJob &J);

__global__ void __launch_bounds__(SCHOOL_THREADS) k_school(const SchoolJob *__restrict__ jobs) {
    const SchoolJob J = jobs[blockIdx.y];
    if (blockIdx.x >= school_ctas(J.nlimbs)) return;
    school_block(J);
}

// Up to two schoolbook products by value (the doubling step's two squarings
// while the operands are short).
struct SchoolPair {
    SchoolJob j[2];
};
__global__ void __launch_bounds__(SCHOOL_THREADS) k_school_pair(SchoolPair P) {
    const SchoolJob &J = P.j[blockIdx.y];
    if (blockIdx.x >= school_ctas(J.nlimbs)) return;
    school_block(J);
}

FFG_DEV_INLINE void school_block(const SchoolJob &J) {
    constexpr uint32_t NC = SCHOOL_NL + 3; // columns j0 - 3 .. j0 + NL - 1
    __shared__ uint64_t t0s[NC], t1s[NC];
    __shared__ uint32_t t2s[NC];
    __shared__ uint64_t lo[SCHOOL_NL];
    __shared__ uint32_t hi[SCHOOL_NL];
    __shared__ uint32_t gG[SCHOOL_NL / 32], gP[SCHOOL_NL / 32], gin[SCHOOL_NL / 32];
    __shared__ uint32_t hiprev_s;
    const int64_t j0 = (int64_t)blockIdx.x * SCHOOL_NL;
    for (uint32_t c = threadIdx.x; c < NC; c += blockDim.x) {
        uint64_t a, b, d;
        school_col(J, j0 - 3 + (int64_t)c, a, b, d);
        t0s[c] = a;
        t1s[c] = b;
        t2s[c] = (uint32_t)d;
    }
    __syncthreads();
    // v_j = t0_j + t1_(j-1) + t2_(j-2), for j = j0 - 1 .. j0 + NL - 1
    for (int32_t jl = (int32_t)threadIdx.x - 1; jl < (int32_t)SCHOOL_NL; jl += blockDim.x) {
        const uint32_t c = (uint32_t)(jl + 3);
        const u128 v = (u128)t0s[c] + t1s[c - 1] + t2s[c - 2];
        if (jl < 0) hiprev_s = (uint32_t)(v >> 64);
        else {
            lo[jl] = (uint64_t)v;
            hi[jl] = (uint32_t)(v >> 64);
        }
    }
    __syncthreads();
    const uint32_t map = cta_resolve(lo, hi, blockIdx.x ? hiprev_s : 0, SCHOOL_NL, gG, gP, gin);
    for (uint32_t j = threadIdx.x; j < SCHOOL_NL && (uint64_t)j0 + j < J.nlimbs; j += blockDim.x) J.out[j0 + j] = lo[j];
    if (threadIdx.x == 0) J.maps[blockIdx.x] = map;
    const uint32_t ncta = school_ctas(J.nlimbs);
    if (ncta > 1 && last_cta(J.ticket, ncta)) {
        settle_cta(J.out, J.nlimbs, SCHOOL_NL, J.maps, ncta);
        if (threadIdx.x == 0) *J.ticket = 0;
    }
}

cudaError_t launch_school_pair(const SchoolJob *jobs, uint32_t count, cudaStream_t st) {
    SchoolPair P{};
    uint32_t mx = 0;
    double bytes = 0;
    for (uint32_t i = 0; i < count && i < 2; i++) {
        P.j[i] = jobs[i];
        mx = max(mx, school_ctas(jobs[i].nlimbs));
        bytes += 8.0 * (double)(jobs[i].na + jobs[i].nb + jobs[i].nlimbs);
    }
    prof_begin(PK_SCHOOL, st);
    k_school_pair<<<dim3(mx, count), SCHOOL_THREADS, 0, st>>>(P);
    prof_end(PK_SCHOOL, st, bytes);
    return cudaGetLastError();
}

// k_school_sq_pair: the doubling step's two short squarings (operands of up
// to a few hundred limbs) spread over more CTAs than k_school_pair gives
// them: SQ_NL = 64 output limbs per CTA, 4 threads per column, and the
// symmetry of a square: column j = 2 sum_{i < j - i} a_i a_(j-i) + a_(j/2)^2
// (j even).  The same 192-bit column sums, ripple settle and last-CTA carry
// settle as k_school.
constexpr uint32_t SQ_NL = 64;
constexpr uint32_t SQ_TPC = 4; // threads per column

__host__ __device__ uint32_t school_sq_ctas(uint64_t nlimbs) { return (uint32_t)((nlimbs + SQ_NL - 1) / SQ_NL); }

__global__ void __launch_bounds__(SCHOOL_THREADS) k_school_sq_pair(SchoolPair Pr) {
    const SchoolJob &J = blockIdx.y ? Pr.j[1] : Pr.j[0];
    const uint32_t ncta = school_sq_ctas(J.nlimbs);
    if (blockIdx.x >= ncta) return;
    constexpr uint32_t NC = SQ_NL + 3; // columns j0 - 3 .. j0 + SQ_NL - 1
    __shared__ uint64_t p0[NC][SQ_TPC], p1[NC][SQ_TPC];
    __shared__ uint32_t p2[NC][SQ_TPC];
    __shared__ uint64_t t0s[NC], t1s[NC];
    __shared__ uint32_t t2s[NC];
    __shared__ uint64_t lo[SQ_NL];
    __shared__ uint32_t hi[SQ_NL];
    __shared__ uint32_t gG[SQ_NL / 32], gP[SQ_NL / 32], gin[SQ_NL / 32];
    __shared__ uint32_t hiprev_s;
    const int64_t j0 = (int64_t)blockIdx.x * SQ_NL, n = (int64_t)J.na;
    const uint64_t *a = J.a;
    // partial sums of a_i a_(j-i) over i < j - i, i = part (mod SQ_TPC)
    for (uint32_t slot = threadIdx.x; slot < NC * SQ_TPC; slot += blockDim.x) {
        const uint32_t c = slot / SQ_TPC, part = slot % SQ_TPC;
        const int64_t j = j0 - 3 + (int64_t)c;
        uint64_t t0 = 0, t1 = 0, t2 = 0;
        if (j >= 1 && j <= 2 * n - 3) {
            const int64_t ilo = j - n + 1 > 0 ? j - n + 1 : 0, ihi = (j - 1) / 2; // i < j - i
            for (int64_t i = ilo + part; i <= ihi; i += SQ_TPC) {
                const u128 pr = (u128)__ldg(&a[i]) * __ldg(&a[j - i]);
                const uint64_t l = (uint64_t)pr, h = (uint64_t)(pr >> 64);
                t0 += l;
                const uint64_t hh = h + (t0 < l);
                t1 += hh;
                t2 += t1 < hh;
            }
        }
        p0[c][part] = t0;
        p1[c][part] = t1;
        p2[c][part] = (uint32_t)t2;
    }
    __syncthreads();
    // column j: 2 S_j + a_(j/2)^2, in 192 bits
    for (uint32_t c = threadIdx.x; c < NC; c += blockDim.x) {
        const int64_t j = j0 - 3 + (int64_t)c;
        uint64_t t0 = 0, t1 = 0, t2 = 0;
        for (uint32_t q = 0; q < SQ_TPC; q++) {
            t0 += p0[c][q];
            const uint64_t c0 = t0 < p0[c][q];
            const uint64_t x1 = p1[c][q] + c0; // p1 < 2^64 - 1 is not assured: carry both ways
            const uint64_t c1 = x1 < c0;
            t1 += x1;
            t2 += p2[c][q] + c1 + (t1 < x1);
        }
        // doubled
        t2 = (t2 << 1) | (t1 >> 63);
        t1 = (t1 << 1) | (t0 >> 63);
        t0 <<= 1;
        if (j >= 0 && j <= 2 * n - 2 && (j & 1) == 0) {
            const uint64_t x = __ldg(&a[j / 2]);
            const u128 sq = (u128)x * x;
            const uint64_t l = (uint64_t)sq, h = (uint64_t)(sq >> 64);
            t0 += l;
            const uint64_t c0 = t0 < l;
            const uint64_t x1 = h + c0;
            const uint64_t c1 = x1 < c0;
            t1 += x1;
            t2 += c1 + (t1 < x1);
        }
        t0s[c] = t0;
        t1s[c] = t1;
        t2s[c] = (uint32_t)t2;
    }
    __syncthreads();
    // v_j = t0_j + t1_(j-1) + t2_(j-2), for j = j0 - 1 .. j0 + SQ_NL - 1
    for (int32_t jl = (int32_t)threadIdx.x - 1; jl < (int32_t)SQ_NL; jl += blockDim.x) {
        const uint32_t c = (uint32_t)(jl + 3);
        const u128 v = (u128)t0s[c] + t1s[c - 1] + t2s[c - 2];
        if (jl < 0) hiprev_s = (uint32_t)(v >> 64);
        else {
            lo[jl] = (uint64_t)v;
            hi[jl] = (uint32_t)(v >> 64);
        }
    }
    __syncthreads();
    const uint32_t map = cta_resolve(lo, hi, blockIdx.x ? hiprev_s : 0, SQ_NL, gG, gP, gin);
    for (uint32_t j = threadIdx.x; j < SQ_NL && (uint64_t)j0 + j < J.nlimbs; j += blockDim.x) J.out[j0 + j] = lo[j];
    if (threadIdx.x == 0) J.maps[blockIdx.x] = map;
    if (ncta > 1 && last_cta(J.ticket, ncta)) {
        settle_cta(J.out, J.nlimbs, SQ_NL, J.maps, ncta);
        if (threadIdx.x == 0) *J.ticket = 0;
    }
}

cudaError_t launch_school_sq_pair(const SchoolJob *jobs, uint32_t count, cudaStream_t st) {
    SchoolPair P{};
    uint32_t mx = 0;
    double bytes = 0;
    for (uint32_t i = 0; i < count && i < 2; i++) {
        if (jobs[i].a != jobs[i].b || jobs[i].na != jobs[i].nb) return cudaErrorInvalidValue;
        P.j[i] = jobs[i];
        mx = max(mx, school_sq_ctas(jobs[i].nlimbs));
        bytes += 8.0 * (double)(jobs[i].na + jobs[i].nlimbs);
    }
    prof_begin(PK_SCHOOL, st);
    k_school_sq_pair<<<dim3(mx, count), SCHOOL_THREADS, 0, st>>>(P);
    prof_end(PK_SCHOOL, st, bytes);
    return cudaGetLastError();
}

cudaError_t launch_school_batch(const SchoolJob *d_jobs, uint32_t count, uint32_t max_ctas, cudaStream_t st,
                                double bytes) {
    if (!count) return cudaSuccess;
    prof_begin(PK_SCHOOL, st);
    k_school<<<dim3(max_ctas, count), SCHOOL_THREADS, 0, st>>>(d_jobs);
    prof_end(PK_SCHOOL, st, bytes);
    return cudaGetLastError();
}

// ------------------------------------------------------------ linear passes

constexpr uint32_t LIN_NL = 2048; // limbs per CTA
constexpr uint32_t LIN_THREADS = 256;

uint32_t lin_ctas(uint64_t len) { return (uint32_t)((len + LIN_NL - 1) / LIN_NL); }

// Column sum of output k at limb j (0 past the output), from the limbs x, y
// of s1, s2 at j.
FFG_DEV_INLINE void lin_colsum(const LinJob &J, uint32_t k, uint64_t j, uint64_t x, uint64_t y, uint64_t &s_lo,
                               uint32_t &s_hi) {
    s_lo = 0;
    s_hi = 0;
    if (j >= J.len) return;
    const int64_t al = k ? J.alpha[1] : J.alpha[0], be = k ? J.beta[1] : J.beta[0];
    const int64_t ga = k ? J.gamma[1] : J.gamma[0];
    const u128 t = (u128)(al >= 0 ? x : ~x) * (uint64_t)(al >= 0 ? al : -al) +
                   (u128)(be >= 0 ? y : ~y) * (uint64_t)(be >= 0 ? be : -be);
    // constant: gamma plus one per negative term (-s = ~s + 1), two's complement
    const int64_t c = ga + (al < 0 ? -al : 0) + (be < 0 ? -be : 0);
    const uint64_t cj = j == 0 ? (uint64_t)c : (c < 0 ? ~0ull : 0ull);
    const u128 sum = t + cj;
    s_lo = (uint64_t)sum;
    s_hi = (uint32_t)(sum >> 64);
}

__global__ void __launch_bounds__(LIN_THREADS) k_lin(LinJob J) {
    __shared__ uint64_t lo[LIN_NL];
    __shared__ uint32_t hi[LIN_NL];
    __shared__ uint32_t gG[LIN_NL / 32], gP[LIN_NL / 32], gin[LIN_NL / 32];
    __shared__ uint32_t hiprev_s;
    constexpr int PER = LIN_NL / LIN_THREADS;
    const uint64_t j0 = (uint64_t)blockIdx.x * LIN_NL;
    // every limb this thread needs, loaded once for both outputs
    uint64_t xs[PER], ys[PER];
#pragma unroll
    for (int r = 0; r < PER; r++) {
        const uint64_t j = j0 + threadIdx.x + r * LIN_THREADS;
        xs[r] = j < J.n1 ? __ldg(&J.s1[j]) : 0;
        ys[r] = j < J.n2 ? __ldg(&J.s2[j]) : 0;
    }
    uint64_t xp = 0, yp = 0; // limb j0 - 1, for the carry into the CTA's first limb
    if (threadIdx.x == 0 && j0 > 0) {
        xp = j0 - 1 < J.n1 ? J.s1[j0 - 1] : 0;
        yp = j0 - 1 < J.n2 ? J.s2[j0 - 1] : 0;
    }
    for (uint32_t k = 0; k < J.nout; k++) {
#pragma unroll
        for (int r = 0; r < PER; r++) {
            const uint32_t jl = threadIdx.x + r * LIN_THREADS;
            uint64_t s_lo;
            uint32_t s_hi;
            lin_colsum(J, k, j0 + jl, xs[r], ys[r], s_lo, s_hi);
            lo[jl] = s_lo;
            hi[jl] = s_hi;
        }
        if (threadIdx.x == 0) {
            uint64_t s_lo = 0;
            uint32_t s_hi = 0;
            if (j0 > 0) lin_colsum(J, k, j0 - 1, xp, yp, s_lo, s_hi);
            hiprev_s = s_hi;
        }
        __syncthreads();
        const uint32_t map = cta_resolve(lo, hi, hiprev_s, LIN_NL, gG, gP, gin);
        uint64_t *o = k ? J.out[1] : J.out[0];
        for (uint32_t j = threadIdx.x; j < LIN_NL && j0 + j < J.len; j += blockDim.x) o[j0 + j] = lo[j];
        if (threadIdx.x == 0) J.maps[(size_t)k * gridDim.x + blockIdx.x] = map;
        __syncthreads();
    }
    if (gridDim.x > 1 && last_cta(J.ticket, gridDim.x)) {
        for (uint32_t k = 0; k < J.nout; k++) settle_cta(k ? J.out[1] : J.out[0], J.len, LIN_NL, J.maps + (size_t)k * gridDim.x, gridDim.x);
        if (threadIdx.x == 0) *J.ticket = 0;
    }
}

cudaError_t launch_lin(const LinJob &J, cudaStream_t st) {
    const uint32_t ncta = lin_ctas(J.len);
    prof_begin(PK_LIN, st);
    k_lin<<<ncta, LIN_THREADS, 0, st>>>(J);
    prof_end(PK_LIN, st, 8.0 * (double)(J.n1 + J.n2) + 8.0 * (double)J.len * J.nout);
    return cudaGetLastError();
}

} // namespace ffg
