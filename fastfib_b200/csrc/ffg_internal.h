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
    uint32_t wc, wc_lg;     // columns per CTA in the column passes (a power of 2 dividing 256)
    uint32_t col_stride;    // shared words per column line
    uint32_t square;
    uint32_t mode;          // RowMode of k_row_conv
    uint64_t mstep;         // M / L
    uint32_t scl[3], scls[3];
    // the launch's primes: [prime0, prime0 + nprimes) (blockIdx.y counts
    // from prime0); all three but for a product sharded by prime
    uint32_t prime0 = 0, nprimes = 3;
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

// The CRT of one product: residues (3 arrays of y_stride words, natural
// order) -> nlimbs limbs at out, plus `add` (a small signed constant).
struct CrtJob {
    const uint32_t *y;
    uint64_t y_stride;
    uint64_t conv;
    uint64_t *out;
    uint64_t nlimbs;
    uint32_t width;
    uint32_t pad;
    int64_t add;
    uint32_t *maps;          // crt_ctas(nlimbs, width) words: each CTA's carry map
    uint32_t *ticket;        // a zero word of the ticket pool (ticket_get)
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
    uint32_t pad;
    uint32_t *maps;          // 2 * lin_ctas(len) words: each CTA's carry map per output
    uint32_t *ticket;        // a zero word of the ticket pool (ticket_get)
};

// The CRT of a fast-doubling step's two squarings fused with its linear
// pass: out_k = alpha_k s1 + beta_k s2 + gamma_k (k = 0, 1, len limbs each)
// straight from the residues of s1 = y[0] and s2 = y[1] (same width and
// length), without writing s1 and s2.
struct CrtLinJob {
    const uint32_t *y[2];
    uint64_t y_stride;
    uint64_t conv[2];
    uint64_t *out[2];
    uint64_t len;
    uint32_t width;
    uint32_t pad;
    int32_t alpha[2], beta[2];
    int64_t gamma[2];
    uint32_t *maps;          // 2 * crt_ctas(len, width) words
    uint32_t *ticket;        // a zero word of the ticket pool (ticket_get)
};

// Jobs travel to the kernels by value, as kernel parameters: nothing is
// copied to the device per launch, so launches queue up without waiting and
// a whole chain can be captured into a CUDA graph.
constexpr int FFG_CONV_JOBS = 2; // one-CTA convolutions per launch
constexpr int FFG_FS_JOBS = 4;   // four-step products (or split pieces) per launch
// A launch takes its jobs inline, or -- for batches of any size -- from a
// device array `ext` (then the inline entries are unused).
struct ConvJobs {
    ConvJob j[FFG_CONV_JOBS];
    const ConvJob *ext;
};
struct FSJobs {
    FSJob j[FFG_FS_JOBS];
    const FSJob *ext;
};

// One schoolbook product out = a b (the reference's big_mul_schoolbook,
// src/bigint.c:257-276), nlimbs = na + nb (+ slack) limbs fully written.
struct SchoolJob {
    const uint64_t *a, *b;
    uint64_t na, nb;
    uint64_t *out;
    uint64_t nlimbs;
    uint32_t *maps; // school_ctas(nlimbs) words
    uint32_t *ticket; // a zero word of the ticket pool (ticket_get)
};

// Carries between the CTAs of one CRT, schoolbook product or linear pass are
// settled inside the same launch: every CTA publishes its carry map, takes a
// ticket (an atomic count on a word that is zero between launches), and the
// CTA that draws the last ticket scans the maps, adds the carries and zeroes
// the word again.  ticket_get hands out distinct words of a pool zeroed once;
// launches captured into CUDA graphs draw from a region of their own.
uint32_t *ticket_get();

// ---------------------------------------------------- decimal conversion jobs

// out = bits [shift, shift + 64 nout) of src (nsrc limbs, zero beyond).
struct ShiftJob {
    const uint64_t *src;
    uint64_t nsrc;
    uint64_t *out;
    uint64_t nout;
    uint64_t shift;
};

// out = sum over t of mul[t] (* *scale[t]) src[t] + add (+ *add_dev), mod
// 2^(64 len); top_bits nonzero: the top limb keeps its low top_bits bits;
// a negative result is one whose top limb ends with bit 63 set.
struct CombJob {
    const uint64_t *src[3];
    uint64_t n[3];              // limbs of each source; 0: term unused
    int32_t mul[3];
    const uint32_t *scale[3];   // nullable
    uint64_t *out;
    uint64_t len;
    int64_t add;
    const uint32_t *add_dev;    // nullable
    uint32_t top_bits;
    uint32_t *neg_flag;         // nullable: raised (atomic or) on a negative result
    uint32_t *sign_out;         // nullable: written 1 / 0 for a negative / non-negative result
    uint32_t *maps;             // comb_ctas(len, nl) words
    uint32_t *ticket;
};

// khat = an estimate of floor((x - qp) / P) for P of s bits, exact or one
// too large; flag raised if the estimate is out of range.
struct KhatJob {
    const uint64_t *x, *qp, *P;
    uint64_t nx, nqp, nP;
    uint64_t s;
    uint32_t *khat;
    uint32_t *flag;
};

// One leaf piece (below 10^(19 chunks)).
constexpr int FFG_LEAF_MAX_LIMBS = 130;
struct LeafJob {
    const uint64_t *x;
    uint64_t n;
};

__host__ __device__ uint32_t comb_nl(uint64_t max_len);           // limbs per CTA of a launch
__host__ __device__ uint32_t comb_ctas(uint64_t len, uint32_t nl);
cudaError_t launch_first_nonzero(const char *d, uint64_t n, unsigned long long *d_first, cudaStream_t st);
cudaError_t launch_shift_batch(const ShiftJob *d_jobs, uint32_t count, uint64_t max_out, cudaStream_t st);
cudaError_t launch_comb_batch(const CombJob *d_jobs, uint32_t count, uint64_t max_len, cudaStream_t st);
cudaError_t launch_khat_batch(const KhatJob *d_jobs, uint32_t count, cudaStream_t st);
cudaError_t launch_leaf_digits(const LeafJob *d_jobs, uint32_t count, uint32_t chunks, uint64_t v, char *d_out,
                               cudaStream_t st);
cudaError_t launch_bit_length(const uint64_t *x, uint64_t n, uint64_t *d_out, cudaStream_t st);

uint32_t crt_ctas(uint64_t nlimbs, uint32_t width); // CTAs (and carry maps) of one CRT
__host__ __device__ uint32_t school_ctas(uint64_t nlimbs); // CTAs (and carry maps) of one schoolbook product
// Batches in device arrays: one launch (plus one settle) for all products.
cudaError_t launch_crt_batch(const CrtJob *d_jobs, uint32_t count, uint32_t max_ctas, cudaStream_t st,
                             double bytes);
// CRTs of different sizes in one launch of total_ctas CTAs: d_first holds the
// count + 1 prefix sums of the jobs' crt_ctas.
cudaError_t launch_crt_flat(const CrtJob *d_jobs, const uint32_t *d_first, uint32_t count, uint32_t total_ctas,
                            cudaStream_t st, double bytes);
cudaError_t launch_school_pair(const SchoolJob *jobs, uint32_t count, cudaStream_t st);
// The doubling step's two short squarings (a == b), SQ_NL output limbs per
// CTA: school_sq_ctas(nlimbs) words of maps each.
cudaError_t launch_school_sq_pair(const SchoolJob *jobs, uint32_t count, cudaStream_t st);
__host__ __device__ uint32_t school_sq_ctas(uint64_t nlimbs); // 1 or 2, by value
cudaError_t launch_school_batch(const SchoolJob *d_jobs, uint32_t count, uint32_t max_ctas, cudaStream_t st,
                                double bytes);
uint32_t lin_ctas(uint64_t len);                    // CTAs of one linear pass

cudaError_t set_line_consts(const LineConsts &h); // once, before any transform
cudaError_t set_line_consts_rows(const LineConsts &h); // the same for ffg_rows.cu
cudaError_t set_line_consts_cols(const LineConsts &h); // and ffg_cols.cu
// The fixed-shape column passes (ffg_cols.cu) for the geometries col2_ok
// accepts; nz is the grid depth (jobs x operands forward, jobs inverse).
bool col2_ok(const FourStep &G);
cudaError_t launch_col2(bool fwd, const Primes3 &P3, const FourStep &G, const FSJobs &jobs, uint32_t nz,
                        cudaStream_t st);
// The fixed-shape row pass (ffg_rows.cu) for the geometries row2_ok accepts.
bool row2_ok(const FourStep &G);
cudaError_t launch_row2(const Primes3 &P3, const FourStep &G, const FSJobs &jobs, uint32_t njobs, cudaStream_t st);
// Load (and configure) the kernels of one product -- the transforms and the
// plain CRT -- during set-up, so a later first launch loads no module code.
cudaError_t ntt_kernels_load();
cudaError_t crt_kernel_load();
cudaError_t launch_conv_small(const Primes3 &P3, const ConvJobs &jobs, uint32_t njobs, uint32_t maxL,
                              bool any_distinct, cudaStream_t st, double bytes);
cudaError_t launch_four_step(const Primes3 &P3, const FourStep &G, const FSJobs &jobs, uint32_t njobs,
                             cudaStream_t st, double limb_bytes);
cudaError_t launch_split_forward(const Primes3 &P3, FourStep G, const FSJobs &jobs, uint32_t njobs,
                                 cudaStream_t st, double limb_bytes);
cudaError_t launch_split_piece(const Primes3 &P3, FourStep G, const FSJob &job, uint32_t pairs, cudaStream_t st);
cudaError_t launch_crt(const Primes3 &P3, const CrtJob &J, cudaStream_t st);
cudaError_t launch_crt_pair(const CrtJob *jobs, uint32_t count, cudaStream_t st); // count 1 or 2, by value
cudaError_t launch_lin(const LinJob &J, cudaStream_t st);
cudaError_t launch_crt_lin(const CrtLinJob &J, cudaStream_t st);

// The cost model's kernels (ffg_mlp.cu); parameters, rows and outputs on the device.
cudaError_t launch_mlp_train(float *d_params, const float *d_X, const int32_t *d_M, const float *d_Y, uint32_t n,
                             uint32_t epochs, float lr, float *d_loss_hist, cudaStream_t st);
cudaError_t launch_mlp_grad(const float *d_params, const float *d_X, const int32_t *d_M, const float *d_Y, uint32_t n,
                            float *d_grad, float *d_loss, cudaStream_t st);
cudaError_t launch_mlp_infer(const float *d_params, const float *d_X, uint32_t n, float *d_out, cudaStream_t st);

// Fingerprints (ffg_fingerprint.cu): x mod each prime into d_out, using
// fingerprint_blocks() * FFG_FP_PRIMES words of partial sums and a zero ticket.
cudaError_t launch_fingerprint(const uint64_t *x, uint64_t n, const uint64_t *primes, uint64_t *partial,
                               uint32_t *ticket, uint64_t *d_out, cudaStream_t st);
uint32_t fingerprint_blocks();
cudaError_t launch_bits_mb(const uint64_t *x, uint64_t n, unsigned long long *d_out, cudaStream_t st);

// Kernel families the profiler tracks (ffg_profile_read in include/ffg.h).
enum ProfKind { PK_CONV_SMALL = 0, PK_COL_FWD, PK_ROW_CONV, PK_COL_INV, PK_CRT, PK_CARRY, PK_LIN, PK_SCHOOL, PK_COUNT };

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
