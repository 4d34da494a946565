// Kernels of the device decimal conversion (the reference's big_to_string,
// src/decimal.c:229-281, breadth first): every piece of one level of the
// divide-and-conquer goes through the same few launches.
//
//   k_shift_batch : out = bits [shift, shift + 64 nout) of src (Barrett's
//                   x >> (s - 1) and t >> (s + 1), Newton's truncations)
//   k_comb_batch  : out = sum of up to three signed, optionally per-job
//                   device-scaled sources plus a constant, mod 2^(64 len)
//                   (Barrett's r = x - q P - k P and q + k, Newton's
//                   2^(2s) - P y and y + c): column sums in two's complement,
//                   ripples by cta_resolve, carries between CTAs settled by the
//                   CTA that finishes last
//   k_khat_batch  : k = floor(r / P) for r = x - q P < 2^5 P from 64-bit
//                   windows of x, q P and P at bit s - 58, biased up so that
//                   k is exact or one too large (then x - q P - k P comes out
//                   negative, and a second combination adds P back)
//   k_leaf_digits : a piece below 10^(19 c) into 19 c digits by c divisions
//                   by 10^19 with a precomputed inverse (division by an
//                   invariant integer, Moller and Granlund, IEEE Trans.
//                   Computers 60(2), 2011, algorithm 4), one thread a piece
//   k_bit_length  : the bit length of one number (the powers' sizes)
#include <cstring>

#include "ffg_internal.h"
#include "ffg_ripple.cuh"

namespace ffg {

typedef unsigned __int128 u128;

// ------------------------------------------------------------------ shift

__global__ void __launch_bounds__(256) k_shift_batch(const ShiftJob *__restrict__ jobs) {
    const ShiftJob J = jobs[blockIdx.y];
    const uint64_t w = J.shift >> 6;
    const uint32_t b = (uint32_t)(J.shift & 63);
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < J.nout; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t k = i + w;
        const uint64_t lo = k < J.nsrc ? J.src[k] : 0, hi = k + 1 < J.nsrc ? J.src[k + 1] : 0;
        J.out[i] = b ? (lo >> b) | (hi << (64 - b)) : lo;
    }
}

cudaError_t launch_shift_batch(const ShiftJob *d_jobs, uint32_t count, uint64_t max_out, cudaStream_t st) {
    if (!count) return cudaSuccess;
    uint64_t blocks = (max_out + 255) / 256;
    if (blocks > 1024) blocks = 1024;
    if (blocks < 1) blocks = 1;
    for (uint32_t base = 0; base < count; base += 65535) {
        const uint32_t cnt = count - base < 65535 ? count - base : 65535;
        prof_begin(PK_LIN, st);
        k_shift_batch<<<dim3((uint32_t)blocks, cnt), 256, 0, st>>>(d_jobs + base);
        prof_end(PK_LIN, st, 16.0 * (double)max_out * cnt);
        cudaError_t e = cudaGetLastError();
        if (e) return e;
    }
    return cudaSuccess;
}

// ------------------------------------------------------------ combination

constexpr uint32_t COMB_NL = 2048; // most limbs per CTA (a launch uses nl = the pieces' size, 32 .. 2048)
constexpr uint32_t COMB_THREADS = 256;

__host__ __device__ uint32_t comb_nl(uint64_t max_len) {
    uint32_t nl = 32;
    while (nl < COMB_NL && nl < max_len) nl <<= 1;
    return nl;
}
__host__ __device__ uint32_t comb_ctas(uint64_t len, uint32_t nl) { return (uint32_t)((len + nl - 1) / nl); }

struct CombTerms {
    uint64_t mag[3]; // |multiplier| after the device scale
    bool neg[3];
    uint64_t c_lo;   // the constant's limb 0 and the limb above it (two's complement)
    uint64_t c_hi;
};

FFG_DEV_INLINE CombTerms comb_terms(const CombJob &J) {
    CombTerms T;
    int64_t c = J.add + (J.add_dev ? (int64_t)*J.add_dev : 0);
#pragma unroll
    for (int t = 0; t < 3; t++) {
        int64_t m = J.n[t] ? J.mul[t] : 0;
        if (J.scale[t]) m *= (int64_t)*J.scale[t];
        T.neg[t] = m < 0;
        T.mag[t] = (uint64_t)(m < 0 ? -m : m);
        if (m < 0) c += -m; // -m s = m (~s) + m over len limbs
    }
    T.c_lo = (uint64_t)c;
    T.c_hi = c < 0 ? ~0ull : 0ull;
    return T;
}

// Column sum of limb j (0 past len).
FFG_DEV_INLINE void comb_colsum(const CombJob &J, const CombTerms &T, uint64_t j, uint64_t &s_lo, uint32_t &s_hi) {
    s_lo = 0;
    s_hi = 0;
    if (j >= J.len) return;
    u128 acc = j == 0 ? (u128)T.c_lo : (u128)T.c_hi;
#pragma unroll
    for (int t = 0; t < 3; t++) {
        if (!T.mag[t]) continue;
        uint64_t v = j < J.n[t] ? __ldg(&J.src[t][j]) : 0;
        if (T.neg[t]) v = ~v;
        acc += (u128)v * T.mag[t];
    }
    s_lo = (uint64_t)acc;
    s_hi = (uint32_t)(acc >> 64);
}

__global__ void __launch_bounds__(COMB_THREADS) k_comb_batch(const CombJob *__restrict__ jobs, uint32_t nl) {
    __shared__ uint64_t lo[COMB_NL];
    __shared__ uint32_t hi[COMB_NL];
    __shared__ uint32_t gG[COMB_NL / 32], gP[COMB_NL / 32], gin[COMB_NL / 32];
    __shared__ uint32_t hiprev_s;
    const CombJob J = jobs[blockIdx.y];
    const uint32_t ncta = comb_ctas(J.len, nl);
    if (blockIdx.x >= ncta) return;
    const CombTerms T = comb_terms(J);
    const uint64_t j0 = (uint64_t)blockIdx.x * nl;
    for (uint32_t jl = threadIdx.x; jl < nl; jl += blockDim.x) {
        uint64_t s_lo;
        uint32_t s_hi;
        comb_colsum(J, T, j0 + jl, s_lo, s_hi);
        lo[jl] = s_lo;
        hi[jl] = s_hi;
    }
    if (threadIdx.x == 0) {
        uint64_t s_lo = 0;
        uint32_t s_hi = 0;
        if (j0 > 0) comb_colsum(J, T, j0 - 1, s_lo, s_hi);
        hiprev_s = s_hi;
    }
    __syncthreads();
    const uint32_t map = cta_resolve(lo, hi, hiprev_s, nl, gG, gP, gin);
    for (uint32_t j = threadIdx.x; j < nl && j0 + j < J.len; j += blockDim.x) J.out[j0 + j] = lo[j];
    if (threadIdx.x == 0) J.maps[blockIdx.x] = map;
    const bool last = ncta > 1 ? last_cta(J.ticket, ncta) : true;
    if (!last) return;
    // thread 0 reads and may rewrite the top limb: every store of the CTA
    // (its own limbs, the settled carries) must be done first
    if (ncta > 1) settle_cta(J.out, J.len, nl, J.maps, ncta); // ends with a barrier
    else __syncthreads();
    if (threadIdx.x == 0) {
        uint64_t top = __ldcg(&J.out[J.len - 1]);
        if (J.neg_flag && (top >> 63)) atomicOr(J.neg_flag, 1u);
        if (J.sign_out) *J.sign_out = (uint32_t)(top >> 63);
        if (J.top_bits) J.out[J.len - 1] = top & ((1ull << J.top_bits) - 1);
        if (ncta > 1) *J.ticket = 0;
    }
}

cudaError_t launch_comb_batch(const CombJob *d_jobs, uint32_t count, uint64_t max_len, cudaStream_t st) {
    if (!count) return cudaSuccess;
    const uint32_t nl = comb_nl(max_len), ctas = comb_ctas(max_len, nl);
    const uint32_t threads = nl < COMB_THREADS ? nl : COMB_THREADS;
    for (uint32_t base = 0; base < count; base += 65535) {
        const uint32_t cnt = count - base < 65535 ? count - base : 65535;
        prof_begin(PK_LIN, st);
        k_comb_batch<<<dim3(ctas, cnt), threads, 0, st>>>(d_jobs + base, nl);
        prof_end(PK_LIN, st, 32.0 * (double)max_len * cnt);
        cudaError_t e = cudaGetLastError();
        if (e) return e;
    }
    return cudaSuccess;
}

// ------------------------------------------------------------ quotient fix

// 64 bits of x starting at bit e (zero past n limbs).
FFG_DEV_INLINE uint64_t window64(const uint64_t *x, uint64_t n, uint64_t e) {
    const uint64_t w = e >> 6;
    const uint32_t b = (uint32_t)(e & 63);
    const uint64_t lo = w < n ? x[w] : 0, hi = w + 1 < n ? x[w + 1] : 0;
    return b ? (lo >> b) | (hi << (64 - b)) : lo;
}

__global__ void __launch_bounds__(256) k_khat_batch(const KhatJob *__restrict__ jobs, uint32_t count) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const KhatJob J = jobs[i];
    const uint64_t e = J.s - 58;
    const uint64_t d = window64(J.x, J.nx, e) - window64(J.qp, J.nqp, e);
    const uint64_t ptop = window64(J.P, J.nP, e);
    const uint64_t k = (d + 2) / ptop;
    if (k > 64) { // r < 2^5 P by construction: a larger estimate means an error upstream
        atomicOr(J.flag, 1u);
        *J.khat = 0;
        return;
    }
    *J.khat = (uint32_t)k;
}

cudaError_t launch_khat_batch(const KhatJob *d_jobs, uint32_t count, cudaStream_t st) {
    if (!count) return cudaSuccess;
    prof_begin(PK_LIN, st);
    k_khat_batch<<<(count + 255) / 256, 256, 0, st>>>(d_jobs, count);
    prof_end(PK_LIN, st, 48.0 * count);
    return cudaGetLastError();
}

// ----------------------------------------------------------------- leaves

constexpr uint64_t kDec19 = 10000000000000000000ull; // 10^19: its top bit is set (normalised)

// (q, r) = (u1 2^64 + u0) divided by d = 10^19, u1 < d, with
// v = floor((2^128 - 1) / d) - 2^64 (Moller and Granlund, algorithm 4).
FFG_DEV_INLINE uint64_t div_2by1(uint64_t u1, uint64_t u0, uint64_t v, uint64_t &r) {
    const uint64_t d = kDec19;
    u128 q = (u128)v * u1;
    q += ((u128)u1 << 64) + u0 + ((u128)1 << 64); // (u1 + 1, u0) added
    uint64_t q1 = (uint64_t)(q >> 64);
    const uint64_t q0 = (uint64_t)q;
    uint64_t rr = u0 - q1 * d;
    if (rr > q0) {
        q1--;
        rr += d;
    }
    if (rr >= d) {
        q1++;
        rr -= d;
    }
    r = rr;
    return q1;
}

__global__ void __launch_bounds__(32) k_leaf_digits(const LeafJob *__restrict__ jobs, uint32_t count, uint32_t chunks,
                                                      uint64_t v, char *out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const LeafJob J = jobs[i];
    uint64_t t[FFG_LEAF_MAX_LIMBS];
    uint32_t n = (uint32_t)(J.n < FFG_LEAF_MAX_LIMBS ? J.n : FFG_LEAF_MAX_LIMBS);
    for (uint32_t k = 0; k < n; k++) t[k] = J.x[k];
    while (n > 0 && t[n - 1] == 0) n--;
    char *o = out + (uint64_t)i * chunks * 19;
    for (uint32_t c = chunks; c-- > 0;) {
        uint64_t rem = 0;
        for (uint32_t k = n; k-- > 0;) t[k] = div_2by1(rem, t[k], v, rem);
        while (n > 0 && t[n - 1] == 0) n--;
        char *p = o + 19 * c;
        for (int j = 18; j >= 0; j--) {
            const uint64_t q10 = rem / 10;
            p[j] = (char)('0' + (rem - 10 * q10));
            rem = q10;
        }
    }
}

cudaError_t launch_leaf_digits(const LeafJob *d_jobs, uint32_t count, uint32_t chunks, uint64_t v, char *d_out,
                               cudaStream_t st) {
    if (!count) return cudaSuccess;
    prof_begin(PK_LIN, st);
    // one thread a leaf, one warp a CTA: the leaves' serial divisions spread
    // over every SM instead of a quarter as many
    k_leaf_digits<<<(count + 31) / 32, 32, 0, st>>>(d_jobs, count, chunks, v, d_out);
    prof_end(PK_LIN, st, (double)count * chunks * 19);
    return cudaGetLastError();
}

// ---------------------------------------------------------- leading zeros

// The first digit that is not '0': each thread scans 16-byte groups (grid
// stride) and stops at its first find, the block keeps its minimum, and one
// atomic per block publishes it.  d is 16-byte aligned.
__global__ void __launch_bounds__(256) k_first_nonzero(const char *d, uint64_t n, unsigned long long *first) {
    __shared__ unsigned long long best;
    if (threadIdx.x == 0) best = ~0ull;
    __syncthreads();
    const uint64_t groups = (n + 15) / 16, stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; g < groups; g += stride) {
        const uint64_t i0 = 16 * g;
        uint4 v;
        if (i0 + 16 <= n) v = *(const uint4 *)(d + i0);
        else {
            unsigned char b[16];
            for (int k = 0; k < 16; k++) b[k] = i0 + k < n ? (unsigned char)d[i0 + k] : (unsigned char)'0';
            memcpy(&v, b, 16);
        }
        const uint32_t w[4] = {v.x, v.y, v.z, v.w};
        int hit = -1;
        for (int k = 0; k < 16 && hit < 0; k++)
            if (((w[k >> 2] >> (8 * (k & 3))) & 0xffu) != (uint32_t)'0') hit = k;
        if (hit >= 0) {
            atomicMin(&best, (unsigned long long)(i0 + hit));
            break;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0 && best != ~0ull) atomicMin(first, best);
}

cudaError_t launch_first_nonzero(const char *d, uint64_t n, unsigned long long *d_first, cudaStream_t st) {
    const uint64_t blocks = (n + 16 * 256 - 1) / (16 * 256);
    k_first_nonzero<<<(uint32_t)(blocks < 592 ? (blocks ? blocks : 1) : 592), 256, 0, st>>>(d, n, d_first);
    return cudaGetLastError();
}

// ------------------------------------------------------------ bit length

// Bit length of x into *d_out: the multi-block scan of ffg_fingerprint.cu
// (one atomic maximum per thread) on a zeroed word.
cudaError_t launch_bit_length(const uint64_t *x, uint64_t n, uint64_t *d_out, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(d_out, 0, 8, st);
    if (e) return e;
    return launch_bits_mb(x, n, (unsigned long long *)d_out, st);
}

} // namespace ffg
