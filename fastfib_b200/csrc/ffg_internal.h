// Internal types shared by the CUDA translation units of the GPU layer.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "ffg_device.cuh"

namespace ffg {

// Shared-memory words of one padded line of length N, rounded so that
// consecutive lines start one bank apart (stride = 1 mod 32).
__host__ __device__ inline uint32_t line_stride(uint32_t N) {
    uint32_t w = N + (N ? (N - 1) / 32 : 0) + 1;
    return ((w + 31) & ~31u) + 1;
}

// One short convolution (k_conv_small): every prime's residues of a*b,
// natural order, y + prime * y_stride, conv words each.
struct ConvJob {
    const uint64_t *a, *b;
    uint64_t na, nb;        // limbs
    uint64_t ca, cb;        // coefficients of width `width`
    uint32_t *y;
    uint64_t y_stride;
    uint32_t L_words;       // transform length, 3^r3 2^n
    uint32_t n, r3, width;
    uint32_t square;
    uint32_t conv;
    uint32_t scl[3], scls[3]; // 2^32 / L mod p (Shoup pairs)
};

// What the row pass does (FourStep::mode).
enum RowMode : uint32_t {
    ROW_CONV = 0,    // forward both operands, pointwise product, inverse
    ROW_FWD = 1,     // forward only, in place (the split's transformed pieces)
    ROW_ACC_INV = 2, // sum of piece products for one output piece, inverse
};

// Geometry of a four-step launch (shared by its jobs).
struct FourStep {
    uint64_t L;             // transform length = R * 2^c
    uint32_t c;             // log2 of the row length C
    uint32_t R, rn, r3;     // column length R = 3^r3 2^rn
    uint32_t wc;            // columns per CTA in the column passes
    uint32_t col_stride;    // shared words per column line
    uint32_t square;
    uint32_t mode;          // RowMode of k_row_conv
    uint64_t mstep;         // M / L
    uint32_t scl[3], scls[3];
};

// One product of a four-step launch.  ya / yb: 3 * L words each (prime-major);
// ya ends holding the scaled convolution in natural order.  The split's
// pieces read digits [off, off + ca) of their operand.  With yacc set, the
// inverse column pass adds its result into yacc[acc_off ..] (per prime
// acc_stride words) instead of writing ya: the split's overlap-add.
struct FSJob {
    const uint64_t *a, *b;
    uint64_t na, nb, ca, cb;
    uint32_t *ya, *yb;
    uint32_t width, pad;
    uint64_t off_a, off_b;
    // ROW_ACC_INV: output piece m = sum_{i+j=m} A_i B_j over transformed pieces
    const uint32_t *pa, *pb;  // piece i at pa + i * piece_stride
    uint64_t piece_stride;
    uint32_t m, ka, kb, psq;  // psq: pb == pa, pairs i <= j counted twice when i < j
    uint32_t *yacc;
    uint64_t acc_off, acc_stride;
};

// A chunk's (or a run of chunks') carry map c_in -> c_out: a step function
// with at most three values (see ffg_carry.cuh).
struct StepFn {
    __int128 tlo, thi;       // c < tlo -> va; tlo <= c < thi -> vb; c >= thi -> vc
    __int128 va, vb, vc;
};

// The CRT of one product: residues (3 arrays of y_stride words, natural
// order) -> nlimbs limbs at out, plus `add` (a small signed constant) at limb 0.
struct CrtJob {
    const uint32_t *y;
    uint64_t y_stride;
    uint64_t conv;
    uint64_t *out;
    uint64_t nlimbs;
    uint32_t width;
    uint32_t nchunks;        // ceil(nlimbs / width): 64 coefficients each
    int64_t add;
    StepFn *pref;            // per chunk: the map of chunks [CTA start, chunk]
    StepFn *cta_fn;          // one per CTA
    __int128 *cta_in;        // carry into each CTA
};

// A linear combination out_k = alpha_k s1 + beta_k s2 + gamma_k over len limbs
// (two outputs at most): the fast-doubling step and the last factors.
struct LinJob {
    const uint64_t *s1, *s2;
    uint64_t n1, n2, len;
    uint64_t *out[2];
    int32_t alpha[2], beta[2];
    int64_t gamma[2];
    uint32_t nout;
    uint32_t nchunks;        // ceil(len / FFG_LIN_K)
    StepFn *pref;            // 2 * nchunks: per output, as CrtJob::pref
    StepFn *cta_fn;          // 2 per CTA
    __int128 *cta_in;        // 2 per CTA
};

constexpr uint32_t FFG_CRT_THREADS = 128; // chunks (of 64 coefficients) per CTA
constexpr uint32_t FFG_LIN_K = 8;         // limbs per thread in the linear kernels
constexpr uint32_t FFG_LIN_THREADS = 256;

cudaError_t launch_conv_small(const Primes3 &P3, const ConvJob *d_jobs, uint32_t njobs, uint32_t maxL,
                              bool any_distinct, cudaStream_t st, double bytes);
cudaError_t launch_four_step(const Primes3 &P3, const FourStep &G, const FSJob *d_jobs, uint32_t njobs,
                             cudaStream_t st, double limb_bytes);
cudaError_t launch_split_forward(const Primes3 &P3, FourStep G, const FSJob *d_jobs, uint32_t njobs,
                                 cudaStream_t st, double limb_bytes);
cudaError_t launch_split_piece(const Primes3 &P3, FourStep G, const FSJob *d_job, uint32_t pairs, cudaStream_t st);
cudaError_t launch_crt(const Primes3 &P3, const CrtJob &J, cudaStream_t st);
cudaError_t launch_lin(const LinJob &J, cudaStream_t st);

// Kernel families the profiler tracks (ffg_profile_read in include/ffg.h).
enum ProfKind { PK_CONV_SMALL = 0, PK_COL_FWD, PK_ROW_CONV, PK_COL_INV, PK_CRT, PK_CARRY, PK_LIN, PK_COUNT };

// Brackets one kernel launch on stream st with CUDA events when profiling is
// on, and counts launches always.  bytes: the launch's algorithmic bytes.
void prof_begin(int kind, cudaStream_t st);
void prof_end(int kind, cudaStream_t st, double bytes);

struct GarnerConst {
    uint32_t p[3];
    uint32_t i12, i12s, i13, i13s, i23, i23s; // p1^-1 mod p2, p1^-1 mod p3, p2^-1 mod p3 (Shoup)
    uint64_t p12;                              // p1 p2
};
GarnerConst garner_const();

} // namespace ffg
