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
#include <cstdlib>

#include "ffg_internal.h"
#include "ffg_lines.cuh"

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

cudaError_t set_line_consts(const LineConsts &h) { return cudaMemcpyToSymbol(c_lines, &h, sizeof h); }

// Calls body<PI>(...) for the CTA's prime (blockIdx.y, counted from first),
// so each prime's constants are compile-time inside the body.
#define FFG_PRIME_DISPATCH_FROM(first, body, ...)                                                      \
    switch (blockIdx.y + (first)) {                                                                  \
    case 0: body<0>(P3.pr[0], __VA_ARGS__); break;                                                   \
    case 1: body<1>(P3.pr[1], __VA_ARGS__); break;                                                   \
    default: body<2>(P3.pr[2], __VA_ARGS__); break;                                                  \
    }

// ------------------------------------------------------------ short lengths

template <int PI>
FFG_DEV_INLINE void conv_small_body(const PrimeDev &P, const ConvJob &J, uint32_t *smem) {
    const uint32_t L = J.L_words, stride = line_stride(L);
    uint32_t *fa = smem, *fb = smem + stride;
    const bool sq = J.square != 0;
    for (uint32_t i = threadIdx.x; i < L; i += kLineThreads) {
        fa[pad_idx(i)] = i < J.ca ? reduce_digit(digit_at(J.a, J.na, i, J.width), P) : 0;
        if (!sq) fb[pad_idx(i)] = i < J.cb ? reduce_digit(digit_at(J.b, J.nb, i, J.width), P) : 0;
    }
    __syncthreads();
    lines_fwd<PI>(smem, sq ? 0 : 1, J.n, J.r3, stride, P);
    for (uint32_t i = threadIdx.x; i < L; i += kLineThreads) {
        const uint32_t x = fa[pad_idx(i)];
        fa[pad_idx(i)] = mo<PI>(x, sq ? x : fb[pad_idx(i)]);
    }
    __syncthreads();
    lines_inv<PI>(smem, 0, J.n, J.r3, stride, P);
    const uint2 sc = make_uint2(J.scl[PI], J.scls[PI]);
    uint32_t *y = J.y + (size_t)PI * J.y_stride;
    for (uint32_t i = threadIdx.x; i < J.conv; i += kLineThreads) y[i] = sh<PI>(fa[pad_idx(i)], sc);
}

__global__ void __launch_bounds__(kLineThreads, kLineMinBlocks) k_conv_small(Primes3 P3, ConvJobs jobs) {
    extern __shared__ uint32_t smem[];
    __shared__ ConvJob J;
    job_to_smem<ConvJobs, ConvJob, FFG_CONV_JOBS>(jobs, blockIdx.x, &J);
    __syncthreads();
    FFG_PRIME_DISPATCH_FROM(0, conv_small_body, J, smem)
}

// ------------------------------------------------------------- four-step
//
// Column tiles: a CTA holds columns [c0, c0 + wc) of all R rows, wc lines of
// length R.  In the load and store loops thread t serves column t mod wc and
// rows t / wc + m (256 / wc), so a warp touches 32 / wc rows of wc
// consecutive words each.

// Position holding frequency k1 after the forward column transform.
FFG_DEV_INLINE uint32_t pos_of(uint32_t k1, uint32_t n, uint32_t r3) {
    if (!r3) return n ? __brev(k1) >> (32 - n) : 0;
    const uint32_t q = k1 % 3, i = k1 / 3;
    return (q << n) + (n ? __brev(i) >> (32 - n) : 0);
}

template <int PI>
FFG_DEV_INLINE void col_fwd_body(const PrimeDev &P, const FourStep &G, const FSJob &J, uint32_t *smem) {
    const uint32_t z = blockIdx.z, op = G.square ? 0 : (z & 1);
    const uint32_t R = G.R, C = 1u << G.c, wc = G.wc, wlg = G.wc_lg, stride = G.col_stride;
    const uint32_t c0 = blockIdx.x * wc;
    const uint64_t *src = op ? J.b : J.a;
    const uint64_t ns = op ? J.nb : J.na, cs = op ? J.cb : J.ca, off = op ? J.off_b : J.off_a;
    const uint32_t c = threadIdx.x & (wc - 1), r0 = threadIdx.x >> wlg, dr = kLineThreads >> wlg;
    uint32_t *col = smem + c * stride;
    tile_digits<PI, 8>(smem, stride, src, ns, cs, off, J.width, C, R, c0, wlg, P);
    __syncthreads();
    lines_fwd<PI>(smem, wlg, G.rn, G.r3, stride, P);
    // twiddle ω_L^(n2 k1) for k1 = r0 + m dr: a running Montgomery product
    const uint32_t n2 = c0 + c;
    uint32_t cur = twm<PI>(P, (uint64_t)n2 * r0 % G.L * G.mstep);
    const uint32_t step = twm<PI>(P, (uint64_t)n2 * dr % G.L * G.mstep);
    uint32_t *y = (op ? J.yb : J.ya) + (size_t)PI * G.L + n2;
    for (uint32_t k1 = r0; k1 < R; k1 += dr) {
        const uint32_t pos = pos_of(k1, G.rn, G.r3);
        y[(size_t)pos * C] = mo<PI>(col[pad_idx(pos)], cur);
        cur = mo<PI>(cur, step);
    }
}

__global__ void __launch_bounds__(kLineThreads, kLineMinBlocks) k_col_fwd(Primes3 P3, FourStep G, FSJobs jobs) {
    extern __shared__ uint32_t smem[];
    __shared__ FSJob J;
    job_to_smem<FSJobs, FSJob, FFG_FS_JOBS>(jobs, G.square ? blockIdx.z : (blockIdx.z >> 1), &J);
    __syncthreads();
    FFG_PRIME_DISPATCH_FROM(G.prime0, col_fwd_body, G, J, smem)
}

// One row (position pos of the column transform) per CTA.  ROW_CONV: forward
// transform of the row of both operands, pointwise product, inverse.
// ROW_FWD: forward transform only (the split's pieces).  ROW_ACC_INV: the
// split's output piece m, sum over i + j = m of A_i B_j on this row
// (src/mul_split.c:62-78), then the inverse.  The inverse rows end with the
// twiddle ω_L^-(n2 k1), a running product along the row.
template <int PI>
FFG_DEV_INLINE void row_body(const PrimeDev &P, const FourStep &G, const FSJob &J, uint32_t *smem) {
    const uint32_t C = 1u << G.c, pos = blockIdx.x;
    const uint32_t stride = line_stride(C);
    const bool sq = G.square != 0;
    const size_t rowoff = (size_t)PI * G.L + (size_t)pos * C;
    uint32_t *ya = J.ya + rowoff;
    uint32_t *yb = sq ? ya : J.yb + rowoff;
    uint32_t *fa = smem, *fb = smem + stride;

    if (G.mode == ROW_ACC_INV) {
        const uint32_t m = J.m;
        const uint32_t i0 = m + 1 > J.kb ? m + 1 - J.kb : 0;
        uint32_t i1 = m < J.ka - 1 ? m : J.ka - 1;
        if (J.psq && i1 > m / 2) i1 = m / 2;
        for (uint32_t t = threadIdx.x; t < C; t += kLineThreads) {
            uint32_t acc = 0;
            for (uint32_t i = i0; i <= i1; i++) {
                const uint32_t j = m - i;
                const uint32_t v = mo<PI>(J.pa[i * J.piece_stride + rowoff + t], J.pb[j * J.piece_stride + rowoff + t]);
                acc = ad<PI>(acc, v);
                if (J.psq && i < j) acc = ad<PI>(acc, v);
            }
            fa[pad_idx(t)] = acc;
        }
        __syncthreads();
    } else {
        line_load<8>(fa, ya, C);
        if (!sq) line_load<8>(fb, yb, C);
        __syncthreads();
        lines_fwd<PI>(smem, sq ? 0 : 1, G.c, 0, stride, P);
        if (G.mode == ROW_FWD) {
            for (uint32_t i = threadIdx.x; i < C; i += kLineThreads) {
                ya[i] = fa[pad_idx(i)];
                if (!sq) yb[i] = fb[pad_idx(i)];
            }
            return;
        }
        for (uint32_t i = threadIdx.x; i < C; i += kLineThreads) {
            const uint32_t x = fa[pad_idx(i)];
            fa[pad_idx(i)] = mo<PI>(x, sq ? x : fb[pad_idx(i)]);
        }
        __syncthreads();
    }
    lines_inv<PI>(smem, 0, G.c, 0, stride, P);
    const uint32_t k1 = freq_of(pos, G.rn, G.r3);
    // ω^-e = ω^(M - E); exponents reduced mod L first
    const uint64_t e0 = (uint64_t)threadIdx.x * k1 % G.L * G.mstep, e1 = (uint64_t)kLineThreads * k1 % G.L * G.mstep;
    uint32_t cur = twm<PI>(P, e0 ? FFG_M - e0 : 0);
    const uint32_t step = twm<PI>(P, e1 ? FFG_M - e1 : 0);
    for (uint32_t i = threadIdx.x; i < C; i += kLineThreads) {
        ya[i] = mo<PI>(fa[pad_idx(i)], cur);
        cur = mo<PI>(cur, step);
    }
}

__global__ void __launch_bounds__(kLineThreads, kLineMinBlocks) k_row_conv(Primes3 P3, FourStep G, FSJobs jobs) {
    extern __shared__ uint32_t smem[];
    __shared__ FSJob J;
    job_to_smem<FSJobs, FSJob, FFG_FS_JOBS>(jobs, blockIdx.z, &J);
    __syncthreads();
    FFG_PRIME_DISPATCH_FROM(G.prime0, row_body, G, J, smem)
}

template <int PI>
FFG_DEV_INLINE void col_inv_body(const PrimeDev &P, const FourStep &G, const FSJob &J, uint32_t *smem) {
    const uint32_t R = G.R, C = 1u << G.c, wc = G.wc, wlg = G.wc_lg, stride = G.col_stride;
    const uint32_t c0 = blockIdx.x * wc;
    const uint32_t c = threadIdx.x & (wc - 1), r0 = threadIdx.x >> wlg, dr = kLineThreads >> wlg;
    uint32_t *col = smem + c * stride;
    uint32_t *y = J.ya + (size_t)PI * G.L + c0 + c;
    tile_load<8>(smem, stride, J.ya + (size_t)PI * G.L + c0, C, R, wlg);
    __syncthreads();
    lines_inv<PI>(smem, wlg, G.rn, G.r3, stride, P);
    const uint2 sc = make_uint2(G.scl[PI], G.scls[PI]);
    if (J.yacc) { // overlap-add of a split output piece
        uint32_t *acc = J.yacc + (size_t)PI * J.acc_stride + J.acc_off + c0 + c;
        for (uint32_t n1 = r0; n1 < R; n1 += dr) {
            const size_t at = (size_t)n1 * C;
            acc[at] = ad<PI>(acc[at], sh<PI>(col[pad_idx(n1)], sc));
        }
        return;
    }
    for (uint32_t n1 = r0; n1 < R; n1 += dr) y[(size_t)n1 * C] = sh<PI>(col[pad_idx(n1)], sc);
}

__global__ void __launch_bounds__(kLineThreads, kLineMinBlocks) k_col_inv(Primes3 P3, FourStep G, FSJobs jobs) {
    extern __shared__ uint32_t smem[];
    __shared__ FSJob J;
    job_to_smem<FSJobs, FSJob, FFG_FS_JOBS>(jobs, blockIdx.z, &J);
    __syncthreads();
    FFG_PRIME_DISPATCH_FROM(G.prime0, col_inv_body, G, J, smem)
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

cudaError_t ntt_kernels_load() { return smem_optin(); }

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

// The fixed-shape row pass (ffg_rows.cu) where it applies; FFG_ROW2=0 keeps
// the generic one (for comparisons).
static const bool g_row2 = [] {
    const char *v = getenv("FFG_ROW2");
    return !(v && v[0] == '0');
}();
// The fixed-shape column passes (ffg_cols.cu) likewise; FFG_COL2=0 keeps the
// generic ones.
static const bool g_col2 = [] {
    const char *v = getenv("FFG_COL2");
    return !(v && v[0] == '0');
}();

// Geometry the four-step kernels support: lines of at least 2 words (a
// stride-1 step has at least radix 2), rows of at least 4 words and column
// tiles of 4..64 words within a row (16-byte row loads), tiles that fit
// shared memory.
static bool four_step_ok(const FourStep &G) {
    return G.c >= 2 && G.c <= (uint32_t)FFG_LINE_LG && G.rn >= 1 && G.wc >= 4 && G.wc <= 64 &&
           G.wc == (1u << G.wc_lg) && G.wc <= (1u << G.c) && (size_t)G.col_stride * G.wc * 4 <= 200 * 1024;
}

cudaError_t launch_four_step(const Primes3 &P3, const FourStep &G, const FSJobs &jobs, uint32_t njobs,
                             cudaStream_t st, double limb_bytes) {
    if (!four_step_ok(G)) return cudaErrorInvalidValue;
    size_t sm_col = (size_t)G.col_stride * G.wc * sizeof(uint32_t);
    size_t sm_row = (size_t)line_stride(1u << G.c) * (G.square ? 1 : 2) * sizeof(uint32_t);
    cudaError_t e = smem_optin();
    if (e) return e;
    const uint32_t C = 1u << G.c, tiles = C / G.wc;
    const uint32_t nops = G.square ? 1 : 2;
    // algorithmic bytes: one 4-byte read and write of every residue per pass
    // (twiddles excluded); the first pass reads limbs instead of residues
    const double res = 3.0 * 4.0 * (double)G.L * njobs;
    const bool col2 = g_col2 && col2_ok(G);
    prof_begin(PK_COL_FWD, st);
    if (col2) {
        e = launch_col2(true, P3, G, jobs, njobs * nops, st);
    } else {
        k_col_fwd<<<dim3(tiles, G.nprimes, njobs * nops), 256, sm_col, st>>>(P3, G, jobs);
        e = cudaGetLastError();
    }
    prof_end(PK_COL_FWD, st, res * nops + limb_bytes);
    if (e) return e;
    prof_begin(PK_ROW_CONV, st);
    if (g_row2 && row2_ok(G)) {
        e = launch_row2(P3, G, jobs, njobs, st);
    } else {
        k_row_conv<<<dim3(G.R, G.nprimes, njobs), 256, sm_row, st>>>(P3, G, jobs);
        e = cudaGetLastError();
    }
    prof_end(PK_ROW_CONV, st, res * (nops + 1));
    if (e) return e;
    prof_begin(PK_COL_INV, st);
    if (col2) {
        e = launch_col2(false, P3, G, jobs, njobs, st);
    } else {
        k_col_inv<<<dim3(tiles, G.nprimes, njobs), 256, sm_col, st>>>(P3, G, jobs);
        e = cudaGetLastError();
    }
    prof_end(PK_COL_INV, st, res * 2);
    return e;
}

// The split multiply's passes, each over a list of jobs sharing geometry G.
static cudaError_t cfg_four_step(const FourStep &G, size_t *sm_col, size_t *sm_row) {
    if (!four_step_ok(G)) return cudaErrorInvalidValue;
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
    if (g_col2 && col2_ok(G)) {
        e = launch_col2(true, P3, G, jobs, njobs, st);
    } else {
        k_col_fwd<<<dim3(tiles, G.nprimes, njobs), 256, sm_col, st>>>(P3, G, jobs);
        e = cudaGetLastError();
    }
    prof_end(PK_COL_FWD, st, res + limb_bytes);
    if (e) return e;
    prof_begin(PK_ROW_CONV, st);
    k_row_conv<<<dim3(G.R, G.nprimes, njobs), 256, sm_row, st>>>(P3, G, jobs);
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
    k_row_conv<<<dim3(G.R, G.nprimes, 1), 256, sm_row, st>>>(P3, G, one);
    prof_end(PK_ROW_CONV, st, res * (2.0 * pairs + 1.0));
    if ((e = cudaGetLastError())) return e;
    prof_begin(PK_COL_INV, st);
    if (g_col2 && col2_ok(G)) {
        e = launch_col2(false, P3, G, one, 1, st);
    } else {
        k_col_inv<<<dim3(tiles, G.nprimes, 1), 256, sm_col, st>>>(P3, G, one);
        e = cudaGetLastError();
    }
    prof_end(PK_COL_INV, st, res * 3.0);
    return e;
}

} // namespace ffg
