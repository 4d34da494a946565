// Fingerprint of a number held on the device: its bit length, its low 64
// bits and its residues modulo four 64-bit primes -- the check format of the
// reference's tests/memrun.c:19-27, computed where the number lives, for
// results too large to download or to recompute on the host.
//
// k_fp_partial: thread t takes a run of consecutive limbs and reduces it by
// Horner's rule from the top, h = h 2^64 + x_i mod p (with 2^64 mod p
// precomputed), then weights it by 2^(64 i0) mod p (i0 its first limb,
// square-and-multiply) and the CTA sums its threads modulo p.  The CTA that
// finishes last (ticket) adds the CTAs' sums.  Products of two residues below
// p < 2^64 are reduced with unsigned 128-bit remainders.
#include "ffg.h"
#include "ffg_internal.h"
#include "ffg_ripple.cuh"

namespace ffg {

typedef unsigned __int128 u128;

constexpr int FP_THREADS = 256;
constexpr int FP_BLOCKS = 592; // 4 CTAs for each of the 148 SMs

struct FpPrimes {
    uint64_t p[FFG_FP_PRIMES];
    uint64_t r64[FFG_FP_PRIMES]; // 2^64 mod p
};

FFG_DEV_INLINE uint64_t mulmod(uint64_t a, uint64_t b, uint64_t p) { return (uint64_t)(((u128)a * b) % p); }
FFG_DEV_INLINE uint64_t addmod(uint64_t a, uint64_t b, uint64_t p) {
    const u128 s = (u128)a + b;
    return (uint64_t)(s >= p ? s - p : s);
}
FFG_DEV_INLINE uint64_t powmod64(uint64_t b, uint64_t e, uint64_t p) {
    uint64_t r = 1 % p;
    while (e) {
        if (e & 1) r = mulmod(r, b, p);
        b = mulmod(b, b, p);
        e >>= 1;
    }
    return r;
}

__global__ void __launch_bounds__(FP_THREADS) k_fp_partial(const uint64_t *__restrict__ x, uint64_t n, FpPrimes P,
                                                           uint64_t *partial, uint32_t *ticket, uint64_t *out) {
    __shared__ uint64_t red[FFG_FP_PRIMES][FP_THREADS];
    __shared__ bool last;
    const uint64_t nthreads = (uint64_t)gridDim.x * FP_THREADS, t = (uint64_t)blockIdx.x * FP_THREADS + threadIdx.x;
    const uint64_t per = (n + nthreads - 1) / nthreads;
    const uint64_t i0 = t * per < n ? t * per : n, i1 = i0 + per < n ? i0 + per : n;
#pragma unroll
    for (int k = 0; k < FFG_FP_PRIMES; k++) {
        const uint64_t p = P.p[k], r64 = P.r64[k];
        uint64_t h = 0;
        for (uint64_t i = i1; i-- > i0;) h = (uint64_t)(((u128)h * r64 + x[i]) % p);
        if (h) h = mulmod(h, powmod64(r64, i0, p), p);
        red[k][threadIdx.x] = h;
    }
    __syncthreads();
    for (int s = FP_THREADS / 2; s; s >>= 1) {
        if (threadIdx.x < (unsigned)s)
            for (int k = 0; k < FFG_FP_PRIMES; k++)
                red[k][threadIdx.x] = addmod(red[k][threadIdx.x], red[k][threadIdx.x + s], P.p[k]);
        __syncthreads();
    }
    if (threadIdx.x < FFG_FP_PRIMES) partial[(size_t)blockIdx.x * FFG_FP_PRIMES + threadIdx.x] = red[threadIdx.x][0];
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    if (threadIdx.x < FFG_FP_PRIMES) {
        const int k = threadIdx.x;
        uint64_t s = 0;
        for (uint32_t b = 0; b < gridDim.x; b++) s = addmod(s, __ldcg(&partial[(size_t)b * FFG_FP_PRIMES + k]), P.p[k]);
        out[k] = s;
    }
    if (threadIdx.x == 0) *ticket = 0;
}

cudaError_t launch_fingerprint(const uint64_t *x, uint64_t n, const uint64_t *primes, uint64_t *partial,
                               uint32_t *ticket, uint64_t *d_out, cudaStream_t st) {
    FpPrimes P;
    for (int k = 0; k < FFG_FP_PRIMES; k++) {
        P.p[k] = primes[k];
        P.r64[k] = (uint64_t)(((u128)1 << 64) % primes[k]);
    }
    k_fp_partial<<<FP_BLOCKS, FP_THREADS, 0, st>>>(x, n, P, partial, ticket, d_out);
    return cudaGetLastError();
}

uint32_t fingerprint_blocks() { return FP_BLOCKS; }

// Bit length of x: every thread finds the top nonzero limb of its run, one
// atomic maximum per thread.
__global__ void __launch_bounds__(FP_THREADS) k_bits_mb(const uint64_t *__restrict__ x, uint64_t n,
                                                        unsigned long long *out) {
    const uint64_t nthreads = (uint64_t)gridDim.x * FP_THREADS, t = (uint64_t)blockIdx.x * FP_THREADS + threadIdx.x;
    const uint64_t per = (n + nthreads - 1) / nthreads;
    const uint64_t i0 = t * per < n ? t * per : n, i1 = i0 + per < n ? i0 + per : n;
    for (uint64_t i = i1; i-- > i0;)
        if (x[i]) {
            atomicMax(out, (unsigned long long)(64 * i + 64 - __clzll(x[i])));
            return;
        }
}

cudaError_t launch_bits_mb(const uint64_t *x, uint64_t n, unsigned long long *d_out, cudaStream_t st) {
    k_bits_mb<<<FP_BLOCKS, FP_THREADS, 0, st>>>(x, n, d_out);
    return cudaGetLastError();
}

} // namespace ffg
