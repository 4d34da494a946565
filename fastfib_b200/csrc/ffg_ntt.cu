// NTT convolution kernels for sm_100a: three primes, lengths L = 2^k and
// 3 2^k, operands read straight from 64-bit limbs.
//
// Short lengths (L <= 2^FFG_LINE_LG words) run one CTA per (product, prime)
// with the whole transform in shared memory: load digits, forward, pointwise,
// inverse, scale (k_conv_small).  This is the reference's in-cache
// convolution (src/ntt_conv.c:205-226, src/ntt_kernels.c:274-295) as one
// kernel, and the batched path of the decimal conversion and uneven streams.
//
// Long lengths use the four-step split L = R x C (C = 2^c contiguous "rows"
// of the residue array, R = 2^r or 3 2^r "columns"):
//   k_col_fwd  : digits of a column tile -> length-R forward transforms down
//                the columns -> twiddle ω_L^(n2 k1) -> residues, row-major
//   k_row_conv : per row: forward length-C transform of both operands,
//                pointwise product, inverse, twiddle ω_L^-(n2 k1)
//   k_col_inv  : inverse length-R transforms down the columns, scale by
//                2^32 / L, natural coefficient order for the CRT
// The reference's top radix-16 passes over column chunks and in-cache
// sub-blocks (src/ntt_conv.c:158-226) play the same roles on the CPU; here
// each pass is one HBM round trip of the residues.
#include "ffg_device.cuh"
#include "ffg_internal.h"

namespace ffg {

// Job i of a by-value job list, staged once in shared memory so its fields
// occupy no registers across the transform (one thread copies it; callers
// synchronize before use).
template <typename L, typename T, int N>
FFG_DEV_INLINE void job_to_smem(const L &list, uint32_t i, T *dst) {
    if (threadIdx.x == 0) {
        if (list.ext) {
            *dst = list.ext[i];
            return;
        }
#pragma unroll
        for (int k = 0; k < N; k++)
            if (i == (uint32_t)k) *dst = list.j[k];
    }
}

// ------------------------------------------------------------ short lengths

__global__ void __launch_bounds__(256, 3) k_conv_small(Primes3 P3, ConvJobs jobs) {
    extern __shared__ uint32_t smem[];
    __shared__ ConvJob J;
    job_to_smem<ConvJobs, ConvJob, FFG_CONV_JOBS>(jobs, blockIdx.x, &J);
    __syncthreads();
    const PrimeDev P = P3.pr[blockIdx.y];
    const uint32_t L = J.L_words, p = P.p;
    const uint32_t stride = line_stride(L);
    uint32_t *fa = smem, *fb = smem + stride;
    const bool sq = J.square != 0;

    for (uint32_t i = threadIdx.x; i < L; i += blockDim.x) {
        fa[pad_idx(i)] = i < J.ca ? reduce_digit(digit_at(J.a, J.na, i, J.width), P) : 0;
        if (!sq) fb[pad_idx(i)] = i < J.cb ? reduce_digit(digit_at(J.b, J.nb, i, J.width), P) : 0;
    }
    __syncthreads();
    LineSet ls{sq ? 1u : 2u, J.n, J.r3, stride};
    lines_forward(smem, ls, P);
    for (uint32_t i = threadIdx.x; i < L; i += blockDim.x) {
        uint32_t x = fa[pad_idx(i)];
        fa[pad_idx(i)] = mont(x, sq ? x : fb[pad_idx(i)], p, P.pinv);
    }
    __syncthreads();
    ls.lines = 1;
    lines_inverse(smem, ls, P);
    const uint32_t scl = J.scl[blockIdx.y], scls = J.scls[blockIdx.y];
    uint32_t *y = J.y + (size_t)blockIdx.y * J.y_stride;
    for (uint32_t i = threadIdx.x; i < J.conv; i += blockDim.x) y[i] = shoup(fa[pad_idx(i)], scl, scls, p);
}

// ------------------------------------------------------------- four-step

// Column tile: columns [c0, c0 + wc) of all R rows, wc lines of length R.
__global__ void __launch_bounds__(256, 3) k_col_fwd(Primes3 P3, FourStep G, FSJobs jobs) {
    extern __shared__ uint32_t smem[];
    const uint32_t z = blockIdx.z, op = G.square ? 0 : (z & 1), jb = G.square ? z : (z >> 1);
    __shared__ FSJob J;
    job_to_smem<FSJobs, FSJob, FFG_FS_JOBS>(jobs, jb, &J);
    __syncthreads();
    const PrimeDev P = P3.pr[blockIdx.y];
    const uint32_t R = G.R, C = 1u << G.c, wc = G.wc, stride = G.col_stride;
    const uint32_t c0 = blockIdx.x * wc;
    const uint64_t *src = op ? J.b : J.a;
    const uint64_t ns = op ? J.nb : J.na, cs = op ? J.cb : J.ca, off = op ? J.off_b : J.off_a;

    for (uint32_t idx = threadIdx.x; idx < R * wc; idx += blockDim.x) {
        uint32_t n1 = idx / wc, c = idx % wc;
        uint64_t i = (uint64_t)n1 * C + c0 + c;
        smem[c * stride + pad_idx(n1)] = i < cs ? reduce_digit(digit_at(src, ns, off + i, J.width), P) : 0;
    }
    __syncthreads();
    LineSet ls{wc, G.rn, G.r3, stride};
    lines_forward(smem, ls, P);
    uint32_t *y = (op ? J.yb : J.ya) + (size_t)blockIdx.y * G.L;
    for (uint32_t idx = threadIdx.x; idx < R * wc; idx += blockDim.x) {
        uint32_t pos = idx / wc, c = idx % wc;
        uint32_t k1 = freq_of(pos, G.rn, G.r3), n2 = c0 + c;
        uint64_t E = (uint64_t)n2 * k1 * G.mstep;
        uint32_t v = smem[c * stride + pad_idx(pos)];
        y[(size_t)pos * C + n2] = mont(v, tw_mont(P, E), P.p, P.pinv);
    }
}

// One row (position pos of the column transform) per CTA.  ROW_CONV: forward
// transform of the row of both operands, pointwise product, inverse.
// ROW_FWD: forward transform only (the split's pieces).  ROW_ACC_INV: the
// split's output piece m, sum over i + j = m of A_i B_j on this row
// (src/mul_split.c:62-78), then the inverse.
__global__ void __launch_bounds__(256, 3) k_row_conv(Primes3 P3, FourStep G, FSJobs jobs) {
    extern __shared__ uint32_t smem[];
    __shared__ FSJob J;
    job_to_smem<FSJobs, FSJob, FFG_FS_JOBS>(jobs, blockIdx.z, &J);
    __syncthreads();
    const PrimeDev P = P3.pr[blockIdx.y];
    const uint32_t C = 1u << G.c, pos = blockIdx.x, p = P.p;
    const uint32_t stride = line_stride(C);
    const bool sq = G.square != 0;
    uint32_t *ya = J.ya + (size_t)blockIdx.y * G.L + (size_t)pos * C;
    const uint32_t *yb = sq ? ya : J.yb + (size_t)blockIdx.y * G.L + (size_t)pos * C;
    uint32_t *fa = smem, *fb = smem + stride;

    if (G.mode == ROW_ACC_INV) {
        const uint64_t rowoff = (size_t)blockIdx.y * G.L + (size_t)pos * C;
        const uint32_t m = J.m;
        const uint32_t i0 = m + 1 > J.kb ? m + 1 - J.kb : 0;
        uint32_t i1 = m < J.ka - 1 ? m : J.ka - 1;
        if (J.psq && i1 > m / 2) i1 = m / 2;
        for (uint32_t t = threadIdx.x; t < C; t += blockDim.x) {
            uint32_t acc = 0;
            for (uint32_t i = i0; i <= i1; i++) {
                const uint32_t j = m - i;
                uint32_t v = mont(J.pa[i * J.piece_stride + rowoff + t], J.pb[j * J.piece_stride + rowoff + t], p,
                                  P.pinv);
                acc = add_mod(acc, v, p);
                if (J.psq && i < j) acc = add_mod(acc, v, p);
            }
            fa[pad_idx(t)] = acc;
        }
        __syncthreads();
    } else {
        for (uint32_t i = threadIdx.x; i < C; i += blockDim.x) {
            fa[pad_idx(i)] = ya[i];
            if (!sq) fb[pad_idx(i)] = yb[i];
        }
        __syncthreads();
        LineSet lf{sq ? 1u : 2u, G.c, 0, stride};
        lines_forward(smem, lf, P);
        if (G.mode == ROW_FWD) {
            for (uint32_t i = threadIdx.x; i < C; i += blockDim.x) {
                ya[i] = fa[pad_idx(i)];
                if (!sq) ((uint32_t *)yb)[i] = fb[pad_idx(i)];
            }
            return;
        }
        for (uint32_t i = threadIdx.x; i < C; i += blockDim.x) {
            uint32_t x = fa[pad_idx(i)];
            fa[pad_idx(i)] = mont(x, sq ? x : fb[pad_idx(i)], p, P.pinv);
        }
        __syncthreads();
    }
    LineSet ls{1u, G.c, 0, stride};
    lines_inverse(smem, ls, P);
    const uint32_t k1 = freq_of(pos, G.rn, G.r3);
    for (uint32_t i = threadIdx.x; i < C; i += blockDim.x) {
        uint64_t E = (uint64_t)i * k1 * G.mstep;
        E = E ? FFG_M - E : 0; // ω^-e = ω^(M - E)
        ya[i] = mont(fa[pad_idx(i)], tw_mont(P, E), p, P.pinv);
    }
}

__global__ void __launch_bounds__(256, 3) k_col_inv(Primes3 P3, FourStep G, FSJobs jobs) {
    extern __shared__ uint32_t smem[];
    __shared__ FSJob J;
    job_to_smem<FSJobs, FSJob, FFG_FS_JOBS>(jobs, blockIdx.z, &J);
    __syncthreads();
    const PrimeDev P = P3.pr[blockIdx.y];
    const uint32_t R = G.R, C = 1u << G.c, wc = G.wc, stride = G.col_stride;
    const uint32_t c0 = blockIdx.x * wc;
    uint32_t *y = J.ya + (size_t)blockIdx.y * G.L;

    for (uint32_t idx = threadIdx.x; idx < R * wc; idx += blockDim.x) {
        uint32_t pos = idx / wc, c = idx % wc;
        smem[c * stride + pad_idx(pos)] = y[(size_t)pos * C + c0 + c];
    }
    __syncthreads();
    LineSet ls{wc, G.rn, G.r3, stride};
    lines_inverse(smem, ls, P);
    const uint32_t scl = G.scl[blockIdx.y], scls = G.scls[blockIdx.y];
    if (J.yacc) { // overlap-add of a split output piece
        uint32_t *acc = J.yacc + (size_t)blockIdx.y * J.acc_stride + J.acc_off;
        for (uint32_t idx = threadIdx.x; idx < R * wc; idx += blockDim.x) {
            uint32_t n1 = idx / wc, c = idx % wc;
            const size_t at = (size_t)n1 * C + c0 + c;
            acc[at] = add_mod(acc[at], shoup(smem[c * stride + pad_idx(n1)], scl, scls, P.p), P.p);
        }
        return;
    }
    for (uint32_t idx = threadIdx.x; idx < R * wc; idx += blockDim.x) {
        uint32_t n1 = idx / wc, c = idx % wc;
        y[(size_t)n1 * C + c0 + c] = shoup(smem[c * stride + pad_idx(n1)], scl, scls, P.p);
    }
}

// ---------------------------------------------------------------- launchers

// Opts every kernel of this file into the device's largest dynamic shared
// memory once; each launch then asks for what it needs.
static cudaError_t smem_optin() {
    static int done = 0;
    if (done) return cudaSuccess;
    int dev = 0, maxsm = 0;
    cudaError_t e;
    if ((e = cudaGetDevice(&dev))) return e;
    if ((e = cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev))) return e;
    const void *ks[] = {(const void *)k_conv_small, (const void *)k_col_fwd, (const void *)k_row_conv,
                        (const void *)k_col_inv};
    for (const void *k : ks) {
        cudaFuncAttributes fa;
        if ((e = cudaFuncGetAttributes(&fa, k))) return e; // static shared memory counts against the limit
        if ((e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      maxsm - (int)fa.sharedSizeBytes)))
            return e;
    }
    done = 1;
    return cudaSuccess;
}

static size_t small_smem_bytes(uint32_t L, bool square) {
    return (size_t)line_stride(L) * (square ? 1 : 2) * sizeof(uint32_t);
}

cudaError_t launch_conv_small(const Primes3 &P3, const ConvJobs &jobs, uint32_t njobs, uint32_t maxL,
                              bool any_distinct, cudaStream_t st, double bytes) {
    size_t sm = small_smem_bytes(maxL, !any_distinct);
    cudaError_t e = smem_optin();
    if (e != cudaSuccess) return e;
    prof_begin(PK_CONV_SMALL, st);
    k_conv_small<<<dim3(njobs, 3, 1), 256, sm, st>>>(P3, jobs);
    prof_end(PK_CONV_SMALL, st, bytes);
    return cudaGetLastError();
}

cudaError_t launch_four_step(const Primes3 &P3, const FourStep &G, const FSJobs &jobs, uint32_t njobs,
                             cudaStream_t st, double limb_bytes) {
    size_t sm_col = (size_t)G.col_stride * G.wc * sizeof(uint32_t);
    size_t sm_row = (size_t)line_stride(1u << G.c) * (G.square ? 1 : 2) * sizeof(uint32_t);
    cudaError_t e = smem_optin();
    if (e) return e;
    const uint32_t C = 1u << G.c, tiles = C / G.wc;
    const uint32_t nops = G.square ? 1 : 2;
    // algorithmic bytes: one 4-byte read and write of every residue per pass
    // (twiddles excluded); the first pass reads limbs instead of residues
    const double res = 3.0 * 4.0 * (double)G.L * njobs;
    prof_begin(PK_COL_FWD, st);
    k_col_fwd<<<dim3(tiles, 3, njobs * nops), 256, sm_col, st>>>(P3, G, jobs);
    prof_end(PK_COL_FWD, st, res * nops + limb_bytes);
    if ((e = cudaGetLastError())) return e;
    prof_begin(PK_ROW_CONV, st);
    k_row_conv<<<dim3(G.R, 3, njobs), 256, sm_row, st>>>(P3, G, jobs);
    prof_end(PK_ROW_CONV, st, res * (nops + 1));
    if ((e = cudaGetLastError())) return e;
    prof_begin(PK_COL_INV, st);
    k_col_inv<<<dim3(tiles, 3, njobs), 256, sm_col, st>>>(P3, G, jobs);
    prof_end(PK_COL_INV, st, res * 2);
    return cudaGetLastError();
}

// The split multiply's passes, each over a list of jobs sharing geometry G.
static cudaError_t cfg_four_step(const FourStep &G, size_t *sm_col, size_t *sm_row) {
    *sm_col = (size_t)G.col_stride * G.wc * sizeof(uint32_t);
    *sm_row = (size_t)line_stride(1u << G.c) * (G.square ? 1 : 2) * sizeof(uint32_t);
    return smem_optin();
}

// Forward transforms of njobs pieces (one operand each, G.square = 1).
cudaError_t launch_split_forward(const Primes3 &P3, FourStep G, const FSJobs &jobs, uint32_t njobs,
                                 cudaStream_t st, double limb_bytes) {
    size_t sm_col, sm_row;
    G.square = 1;
    G.mode = ROW_FWD;
    cudaError_t e = cfg_four_step(G, &sm_col, &sm_row);
    if (e) return e;
    const uint32_t tiles = (1u << G.c) / G.wc;
    const double res = 3.0 * 4.0 * (double)G.L * njobs;
    prof_begin(PK_COL_FWD, st);
    k_col_fwd<<<dim3(tiles, 3, njobs), 256, sm_col, st>>>(P3, G, jobs);
    prof_end(PK_COL_FWD, st, res + limb_bytes);
    if ((e = cudaGetLastError())) return e;
    prof_begin(PK_ROW_CONV, st);
    k_row_conv<<<dim3(G.R, 3, njobs), 256, sm_row, st>>>(P3, G, jobs);
    prof_end(PK_ROW_CONV, st, res * 2);
    return cudaGetLastError();
}

// One output piece: pairwise sum + inverse row pass, then the inverse column
// pass adding into the whole product's residues.  pairs: products summed.
cudaError_t launch_split_piece(const Primes3 &P3, FourStep G, const FSJob &job, uint32_t pairs, cudaStream_t st) {
    FSJobs one{};
    one.j[0] = job;
    size_t sm_col, sm_row;
    G.square = 1;
    G.mode = ROW_ACC_INV;
    cudaError_t e = cfg_four_step(G, &sm_col, &sm_row);
    if (e) return e;
    const uint32_t tiles = (1u << G.c) / G.wc;
    const double res = 3.0 * 4.0 * (double)G.L;
    prof_begin(PK_ROW_CONV, st);
    k_row_conv<<<dim3(G.R, 3, 1), 256, sm_row, st>>>(P3, G, one);
    prof_end(PK_ROW_CONV, st, res * (2.0 * pairs + 1.0));
    if ((e = cudaGetLastError())) return e;
    prof_begin(PK_COL_INV, st);
    k_col_inv<<<dim3(tiles, 3, 1), 256, sm_col, st>>>(P3, G, one);
    prof_end(PK_COL_INV, st, res * 3.0);
    return cudaGetLastError();
}

} // namespace ffg
