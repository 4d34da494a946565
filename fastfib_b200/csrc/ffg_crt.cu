// CRT recombination and carry propagation for sm_100a.
//
// k_crt_chunks: each thread turns 64 consecutive coefficients into exactly
// `width` limbs.  Per coefficient, Garner's method on the three residues
//   x2 = (r2 - r1) p1^-1 mod p2,  x3 = ((r3 - r1) p1^-1 - x2) p2^-1 mod p3,
//   X  = r1 + x2 p1 + x3 p1 p2  < p1 p2 p3 < 2^93,
// then X is added at bit i*width with a running 128-bit carry (the
// reference's crt_garner8 / crt_pack64, src/crt.c:38-87).  The CTA stages its
// 3 x 8192 residues in shared memory (row pad of one word per 64, so the 32
// threads of a warp reading their own runs hit 32 different banks), writes
// limbs with carry-in 0 and publishes its chunks' carry maps (ffg_carry.cuh).
// k_scan_ctas and k_apply_carry then settle the carries between chunks.
#include "ffg_carry.cuh"
#include "ffg_internal.h"

namespace ffg {

constexpr uint32_t CRT_COEF = 64 * FFG_CRT_THREADS;          // coefficients per CTA
constexpr uint32_t CRT_ROW = CRT_COEF + CRT_COEF / 64;       // padded words per prime

__global__ void __launch_bounds__(FFG_CRT_THREADS) k_crt_chunks(GarnerConst K, CrtJob J) {
    extern __shared__ uint32_t res[];
    __shared__ StepFn wt[FFG_CRT_THREADS / 32];
    const uint64_t gbase = (uint64_t)blockIdx.x * CRT_COEF;
    for (int k = 0; k < 3; k++) {
        const uint32_t *y = J.y + (size_t)k * J.y_stride;
        for (uint32_t i = threadIdx.x; i < CRT_COEF; i += blockDim.x) {
            uint64_t g = gbase + i;
            res[k * CRT_ROW + i + (i >> 6)] = g < J.conv ? y[g] : 0;
        }
    }
    __syncthreads();

    const uint32_t t = threadIdx.x;
    const uint64_t chunk = (uint64_t)blockIdx.x * FFG_CRT_THREADS + t;
    StepFn f = const_fn(0);
    if (chunk < J.nchunks) {
        const uint32_t b = J.width, p1 = K.p[0], p2 = K.p[1], p3 = K.p[2];
        const uint64_t mask = (1ull << b) - 1;
        const uint64_t start = chunk * b;
        const uint64_t lim = J.nlimbs - start; // limbs of this chunk inside the output
        uint64_t *out = J.out + start;
        u128 carry = 0, buf = 0;
        uint32_t nbits = 0, e = 0;
        uint64_t l0 = 0, l1 = 0;
        bool ones = true, zero = true;
        const uint32_t *r = res + 65 * t;
        for (int k = 0; k < 64; k++) {
            uint32_t r1 = r[k], r2 = r[CRT_ROW + k], r3 = r[2 * CRT_ROW + k];
            uint32_t x1m2 = min(r1, r1 - p2);
            uint32_t x2 = shoup(r2 - x1m2 + p2, K.i12, K.i12s, p2);
            uint32_t x1m3 = min(r1, r1 - p3);
            uint32_t t3 = shoup(r3 - x1m3 + p3, K.i13, K.i13s, p3);
            uint32_t x2m3 = min(x2, x2 - p3);
            uint32_t x3 = shoup(t3 - x2m3 + p3, K.i23, K.i23s, p3);
            u128 X = (u128)((uint64_t)x2 * p1 + r1) + (u128)x3 * K.p12;
            u128 acc = X + carry;
            uint64_t v = (uint64_t)acc & mask;
            carry = acc >> b;
            buf |= (u128)v << nbits;
            nbits += b;
            if (nbits >= 64) {
                uint64_t limb = (uint64_t)buf;
                buf >>= 64;
                nbits -= 64;
                if (e < lim) out[e] = limb;
                if (e == 0) l0 = limb;
                else if (e == 1) l1 = limb;
                else {
                    ones &= limb == ~0ull;
                    zero &= limb == 0;
                }
                e++;
            }
        }
        f = chunk_fn((i128)carry, ((u128)l1 << 64) | l0, ones, zero);
    }
    StepFn I = cta_scan(f, wt);
    if (chunk < J.nchunks) J.pref[chunk] = I;
    if (t == blockDim.x - 1) J.cta_fn[blockIdx.x] = I;
}

// One warp: the carry into every CTA from the CTAs' maps and the carry into
// the first one.  Lane l composes a contiguous run of maps, the lanes scan
// their runs, then each lane walks its run once more writing carries.
__global__ void __launch_bounds__(32) k_scan_ctas(const StepFn *__restrict__ fn, uint32_t n, int64_t c0,
                                                  __int128 *__restrict__ cin) {
    const uint32_t lane = threadIdx.x;
    const uint32_t seg = (n + 31) / 32, s0 = min(n, lane * seg), s1 = min(n, s0 + seg);
    StepFn F = const_fn(0);
    if (s0 < s1) {
        F = fn[s0];
        for (uint32_t k = s0 + 1; k < s1; k++) F = fn_then(F, fn[k]);
    }
    // inclusive scan over lanes (empty runs only at the tail, never read)
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        StepFn G = shfl_up_fn(F, d);
        if ((int)lane >= d) F = fn_then(G, F);
    }
    StepFn prev = shfl_up_fn(F, 1);
    i128 c = lane == 0 ? (i128)c0 : fn_apply(prev, (i128)c0);
    for (uint32_t k = s0; k < s1; k++) {
        cin[k] = c;
        c = fn_apply(fn[k], c);
    }
}

// Adds each chunk's carry-in (from its CTA's carry-in and the stored prefix
// map of the chunks before it) into its lowest limbs.
__global__ void __launch_bounds__(256) k_apply_carry(uint64_t *out, uint64_t nlimbs, uint32_t chunk_limbs,
                                                     uint32_t nchunks, uint32_t cta_chunks,
                                                     const StepFn *__restrict__ pref,
                                                     const __int128 *__restrict__ cta_in) {
    const uint64_t chunk = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (chunk >= nchunks) return;
    const uint64_t cta = chunk / cta_chunks;
    i128 c = cta_in[cta];
    if (chunk % cta_chunks) c = fn_apply(pref[chunk - 1], c);
    const uint64_t start = chunk * chunk_limbs;
    const uint64_t n = min((uint64_t)chunk_limbs, nlimbs - start);
    add_carry_in(out + start, n, c);
}

cudaError_t launch_scan_apply(uint64_t *out, uint64_t nlimbs, uint32_t chunk_limbs, uint32_t nchunks,
                              uint32_t cta_chunks, const StepFn *pref, const StepFn *cta_fn, __int128 *cta_in,
                              int64_t c0, cudaStream_t st) {
    const uint32_t ncta = (nchunks + cta_chunks - 1) / cta_chunks;
    prof_begin(PK_CARRY, st);
    k_scan_ctas<<<1, 32, 0, st>>>(cta_fn, ncta, c0, cta_in);
    cudaError_t e = cudaGetLastError();
    if (e) return e;
    k_apply_carry<<<(nchunks + 255) / 256, 256, 0, st>>>(out, nlimbs, chunk_limbs, nchunks, cta_chunks, pref, cta_in);
    prof_end(PK_CARRY, st, (double)nchunks * (sizeof(StepFn) + 32));
    return cudaGetLastError();
}

cudaError_t launch_crt(const Primes3 &P3, const CrtJob &J, cudaStream_t st) {
    (void)P3;
    static bool configured = false;
    const size_t sm = 3 * CRT_ROW * sizeof(uint32_t);
    if (!configured) {
        cudaError_t e = cudaFuncSetAttribute(k_crt_chunks, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e) return e;
        configured = true;
    }
    const uint32_t ncta = (J.nchunks + FFG_CRT_THREADS - 1) / FFG_CRT_THREADS;
    prof_begin(PK_CRT, st);
    k_crt_chunks<<<ncta, FFG_CRT_THREADS, sm, st>>>(garner_const(), J);
    prof_end(PK_CRT, st, 12.0 * (double)J.conv + 8.0 * (double)J.nlimbs);
    cudaError_t e = cudaGetLastError();
    if (e) return e;
    return launch_scan_apply(J.out, J.nlimbs, J.width, J.nchunks, FFG_CRT_THREADS, J.pref, J.cta_fn, J.cta_in,
                             J.add, st);
}

// ------------------------------------------------------------ linear passes

// out_k = alpha_k s1 + beta_k s2 (+ gamma_k, fed in as the first carry) over
// len limbs, FFG_LIN_K limbs per thread: the reference's step_proc and
// last_proc (src/fib.c:37-62, 123-143) with parallel carries.
__global__ void __launch_bounds__(FFG_LIN_THREADS) k_lin_chunks(LinJob J) {
    __shared__ StepFn wt[FFG_LIN_THREADS / 32];
    const uint64_t chunk = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t start = chunk * FFG_LIN_K;
    const uint32_t ncta = gridDim.x;
    for (uint32_t k = 0; k < J.nout; k++) {
        StepFn f = const_fn(0);
        if (chunk < J.nchunks) {
            const i128 al = J.alpha[k], be = J.beta[k];
            uint64_t *o = J.out[k];
            i128 c = 0;
            uint64_t l0 = 0, l1 = 0;
            bool ones = true, zero = true;
#pragma unroll
            for (uint32_t i = 0; i < FFG_LIN_K; i++) {
                const uint64_t idx = start + i;
                const uint64_t x = idx < J.n1 ? J.s1[idx] : 0, y = idx < J.n2 ? J.s2[idx] : 0;
                i128 v = al * (i128)x + be * (i128)y + c;
                const uint64_t limb = (uint64_t)v;
                c = v >> 64;
                if (idx < J.len) o[idx] = limb;
                if (i == 0) l0 = limb;
                else if (i == 1) l1 = limb;
                else {
                    ones &= limb == ~0ull;
                    zero &= limb == 0;
                }
            }
            f = chunk_fn(c, ((u128)l1 << 64) | l0, ones, zero);
        }
        StepFn I = cta_scan(f, wt);
        if (chunk < J.nchunks) J.pref[(size_t)k * J.nchunks + chunk] = I;
        if (threadIdx.x == blockDim.x - 1) J.cta_fn[(size_t)k * ncta + blockIdx.x] = I;
    }
}

cudaError_t launch_lin(const LinJob &J, cudaStream_t st) {
    const uint32_t ncta = (J.nchunks + FFG_LIN_THREADS - 1) / FFG_LIN_THREADS;
    prof_begin(PK_LIN, st);
    k_lin_chunks<<<ncta, FFG_LIN_THREADS, 0, st>>>(J);
    prof_end(PK_LIN, st, 8.0 * (double)(J.n1 + J.n2) + 8.0 * (double)J.len * J.nout);
    cudaError_t e = cudaGetLastError();
    if (e) return e;
    for (uint32_t k = 0; k < J.nout; k++) {
        e = launch_scan_apply(J.out[k], J.len, FFG_LIN_K, J.nchunks, FFG_LIN_THREADS, J.pref + (size_t)k * J.nchunks,
                              J.cta_fn + (size_t)k * ncta, J.cta_in + (size_t)k * ncta, J.gamma[k], st);
        if (e) return e;
    }
    return cudaSuccess;
}

} // namespace ffg
