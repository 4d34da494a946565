/*
 * ffg.h -- the thin C ABI of the B200 layer (libfastfib_b200.so).
 *
 * Plain C types only: sizes, limb pointers (little-endian 64-bit limbs, as
 * the reference's Big, src/common.h:29-33) and an opaque stream handle
 * (a cudaStream_t, or NULL for the library's own stream).  Every function
 * returns 0 on success and a nonzero FFG_E* code on failure; ffg_last_error()
 * then describes the failure.  Calls are serialized by one lock, so the host
 * surface may call in from several threads (the reference calls big_sqr from
 * two pool tasks at once, src/fib.c:184-198).
 *
 * The entry points replace the reference's internal NTT interface; each
 * comment names the reference function whose job it takes over.
 */
#ifndef FFG_H
#define FFG_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    FFG_OK = 0,
    FFG_E_CUDA = 1,     /* a CUDA runtime call failed */
    FFG_E_NOMEM = 2,    /* device or host allocation failed */
    FFG_E_ARG = 3,      /* invalid argument (size, width, length) */
    FFG_E_NODEV = 4,    /* no CUDA device */
    FFG_E_RANGE = 5     /* a size past what this entry point supports */
};

/* The plan of one NTT product: what big_mul_ntt (src/mul_ntt.c:97-118) or the
   split (src/mul_split.c:149-177) would choose, plus the GPU geometry. */
typedef struct {
    uint32_t width;   /* coefficient bits b, 32..35 (split: 8..35) */
    uint32_t lg;      /* transform length L = 2^lg, or 3 * 2^lg when r3 */
    uint32_t r3;
    uint32_t split;   /* 1: piecewise split multiply */
    uint64_t L;       /* transform length (split: the piece length Lp) */
    uint64_t conv;    /* product coefficients ca + cb - 1 */
    uint64_t ca, cb;
    uint64_t ka, kb;  /* split: pieces per operand */
    uint64_t Lbig;    /* split: (ka + kb) * Lp / 2 */
    uint32_t kernel;  /* 0: one-CTA transform, 1: four-step */
    uint32_t row_lg;  /* four-step: log2 of the row length */
} ffg_plan;

/* ntt_init (src/ntt_tables.c:72): sizes the transform cap for products of up
   to max_limbs limbs (2^k >= 2 max_limbs, at most 2^25) and builds the device
   tables on first use.  The cap only grows. */
int ffg_init(size_t max_limbs);
/* g_ntt_max_L (src/mul_basic.c:26): read and override the transform cap (the
   reference's tests set it to force paths, tests/nttfuzz.c:33-39). */
size_t ffg_ntt_max_L(void);
void ffg_set_ntt_max_L(size_t L);
/* NTT_MAX_LG (src/common.h:46-48) at run time: the longest transform 2^lg
   (4..25, default 25); lower values send long products to the split
   multiply, as the reference's -DNTT_MAX_LG builds do (tests/test.ps1:29). */
int ffg_set_max_lg(int lg);
/* big_mul_ntt's choice of width, length and split (src/mul_ntt.c:97-118). */
int ffg_plan_select(uint64_t bits_a, uint64_t bits_b, int square, ffg_plan *plan);

/* big_mul_ntt (src/mul_ntt.c:97) on host limbs: out receives na + nb limbs
   at most (normalized length in *nout).  square != 0 multiplies a by itself
   (the reference signals it by a == b). */
int ffg_mul_host(uint64_t *out, size_t *nout, const uint64_t *a, size_t na, const uint64_t *b, size_t nb,
                 int square);
/* big_mul_ntt on device limbs.  bits_a / bits_b: bit lengths (upper bounds
   are allowed; leading zero limbs are fine).  out: na + nb + 1 limbs of
   device memory, fully written.  stream: a cudaStream_t, or NULL for the
   library's own stream (non-blocking: not ordered after work on the legacy
   default stream). */
int ffg_mul_device(uint64_t *out, const uint64_t *a, size_t na, uint64_t bits_a, const uint64_t *b, size_t nb,
                   uint64_t bits_b, int square, void *stream);

/* Methods for one product of a batch. */
enum {
    FFG_M_PLAIN = -1,   /* the reference's thresholds (src/mul_basic.c:30-38): schoolbook up to
                           64 limbs, the NTT plan of big_mul_ntt from 200 limbs; the range between,
                           Karatsuba over schoolbook in the reference, is one schoolbook product */
    FFG_M_SCHOOL = 0,   /* schoolbook (big_mul_schoolbook, src/bigint.c:257-276) */
    FFG_M_NTT = 1,      /* big_mul_ntt's plan (src/mul_ntt.c:97-118), the split past the cap */
    FFG_M_NTT_POW2 = 2, /* the same width, the transform length forced to 2^k */
    FFG_M_NTT_R3 = 3,   /* the same width, the transform length forced to 3 * 2^k */
    FFG_M_LEARNED = 4   /* the method of least predicted cost under the installed cost model
                           (ffg_mlp_set) among FFG_M_SCHOOL..FFG_M_NTT_R3, taken only when
                           predicted at least 10% cheaper than FFG_M_PLAIN's method; FFG_M_PLAIN
                           without a model, and for products past the transform cap (the split) */
};

/* One product of a batch.  Device variant: a, b, out device pointers, out
   holds na + nb + 1 limbs and is fully written, bits_* are bit lengths (upper
   bounds allowed).  Host variant: host pointers, out holds na + nb limbs,
   bits_* ignored, the normalized length comes back in nout. */
typedef struct {
    const uint64_t *a, *b;
    uint64_t na, nb;
    uint64_t bits_a, bits_b;
    uint64_t *out;
    uint64_t nout;
    int32_t square;
    int32_t method;
} ffg_job;

/* A batch of independent products in as few launches as their plans allow:
   every schoolbook product in one launch, every group of products sharing
   an NTT plan in one launch set and one CRT launch (the reference multiplies
   them one by one, e.g. the products of one decimal level,
   src/decimal.c:177-203). */
int ffg_mul_batch_device(ffg_job *jobs, size_t count, void *stream);
int ffg_mul_batch_host(ffg_job *jobs, size_t count);

/* The learned cost model (no counterpart in the reference, which dispatches
   by fixed thresholds, src/mul_basic.c:30-38): an FP32 MLP
     FFG_MLP_D features -> FFG_MLP_H (tanh) -> FFG_MLP_H (tanh) -> FFG_MLP_K
   whose output m is the predicted log2 microseconds per product of method m
   (FFG_M_SCHOOL .. FFG_M_NTT_R3) inside a batch.  Parameters, in order:
   W1[H][D] b1[H] W2[H][H] b2[H] W3[K][H] b3[K].  Training, gradient and
   inference run in CUDA kernels; a training row is (features, method,
   measured log2 us), the loss half the mean squared error of the row's
   method output. */
#define FFG_MLP_D 8
#define FFG_MLP_H 32
#define FFG_MLP_K 4
#define FFG_MLP_NPARAM                                                                                 \
    (FFG_MLP_H * FFG_MLP_D + FFG_MLP_H + FFG_MLP_H * FFG_MLP_H + FFG_MLP_H + FFG_MLP_K * FFG_MLP_H + FFG_MLP_K)
/* The features of a product of bit lengths bits_a, bits_b (host only). */
int ffg_mlp_features(uint64_t bits_a, uint64_t bits_b, int square, float *f);
/* Trains params (in: initial values, out: trained) on n rows for `epochs`
   full-batch Adam steps of rate lr; loss_hist (NULL or epochs floats) gets the
   loss before each step. */
int ffg_mlp_train(float *params, const float *X, const int32_t *method, const float *y, size_t n, int epochs,
                  float lr, float *loss_hist);
/* One full-batch gradient (FFG_MLP_NPARAM floats) and the loss. */
int ffg_mlp_grad(const float *params, const float *X, const int32_t *method, const float *y, size_t n, float *grad,
                 float *loss);
/* Every output for n feature rows (n * FFG_MLP_K floats); params NULL: the
   installed model. */
int ffg_mlp_predict(const float *params, const float *X, size_t n, float *out);
/* Installs params for FFG_M_LEARNED (copied; sent to the GPU on first use,
   so it works before any device exists); NULL removes the model. */
int ffg_mlp_set(const float *params);
/* Device milliseconds of the launches of one ffg_mul_batch_device call on
   `jobs`: planned and uploaded once, its launches captured as a CUDA graph
   and replayed reps times after one warm-up (the autotuner's clock; the
   host's planning is not timed).  Products past the transform cap (the
   split) are refused. */
int ffg_time_batch(ffg_job *jobs, size_t count, int reps, double *ms);

/* Decimal digits (big_to_string, src/decimal.c:229-281) of a number on the
   device (x: device pointer) or on the host (x: host pointer), converted on
   the device level by level: every level's Barrett products in shared
   launches.  *out is a NUL-terminated string of *nout digits in one of this
   layer's pooled pinned buffers: return it with ffg_free().  *done = 0 when the device path declines -- numbers below
   about 10^4900 and a quotient correction out of range (which its bounds
   rule out) --
   and the caller converts another way (big_to_string then uses its host
   path). */
int ffg_to_decimal_device(const uint64_t *x, size_t nx, char **out, size_t *nout, int *done);
int ffg_to_decimal_host(const uint64_t *x, size_t nx, char **out, size_t *nout, int *done);

/* big_to_string's output streamed (the command line's digit output,
   src/main.c:88-102): the decimal digits of the host number x (nx limbs)
   handed to sink in consecutive pieces, most significant first, leading zeros
   dropped; each piece is valid only during its call.  The leaves of the
   conversion run in slices, and a slice's digits go to the sink while the GPU
   still computes and copies the ones after it.  *ndigits: the digits
   emitted; *done 0 (nothing emitted) when the device path declined -- numbers
   below 10^2432, or a correction out of range -- and the caller converts
   another way (big_to_string).  Zero emits nothing, *done 0. */
typedef void (*ffg_digit_sink)(const char *digits, size_t n, void *user);
int ffg_to_decimal_stream(const uint64_t *x, size_t nx, ffg_digit_sink sink, void *user, size_t *ndigits,
                          int *done);
/* Device milliseconds of the last conversion's levels and leaves (CUDA
   events; the powers, reciprocals and copies excluded). */
double ffg_last_decimal_ms(void);
/* Drops the powers of ten and reciprocals the conversion keeps on the device
   between calls (the next conversion recomputes them). */
void ffg_decimal_cache_clear(void);

/* Fingerprint of a number for checks on results too large to download or to
   recompute (the format of the reference's tests/memrun.c:19-27): out[0] its
   bit length, out[1] its low 64 bits, out[2 + k] its residue modulo
   ffg_fp_primes[k] (18446744073709551557, 18446744073709551533,
   9223372036854775783, 4611686018427387847).  Computed on the device; x a
   device pointer (_device) or a host pointer (_host, copied in). */
#define FFG_FP_PRIMES 4
int ffg_fingerprint_device(const uint64_t *x, size_t n, uint64_t out[2 + FFG_FP_PRIMES]);
int ffg_fingerprint_host(const uint64_t *x, size_t n, uint64_t out[2 + FFG_FP_PRIMES]);

/* Words of the in-launch carry-settle ticket pool that are not zero (0 when
   the GPU is idle; a diagnostic). */
int64_t ffg_tickets_in_use(void);

/* Tuned four-step geometry for transform length 2^lg (r3 0) or 3 * 2^lg
   (r3 1): rows of 2^row_lg words and column tiles of wc columns (the
   reference's fixed pass shapes, src/ntt_conv.c:158-226, have no tuned
   counterpart).  row_lg = wc = 0 restores the default rule.  Captured
   chains are dropped (they hold the old launches). */
int ffg_set_geometry(uint32_t lg, uint32_t r3, uint32_t row_lg, uint32_t wc);
/* The geometry in force for that length. */
int ffg_get_geometry(uint32_t lg, uint32_t r3, uint32_t *row_lg, uint32_t *wc);
/* Loads an autotuner file: lines "geometry lg r3 row_lg wc" and one line
   "mlp N p0 .. p(N-1)" (the cost model, installed as by ffg_mlp_set);
   "#" starts a comment. */
int ffg_load_tuning(const char *path);

/* No counterpart in the reference.  ffg_mul_device without any device
   allocation, for callers that cannot allocate once running: host programs
   whose device memory is all owned by another allocator (a framework's
   caching allocator, a fixed budget handed out at start-up) and
   latency-critical paths that cannot take a cudaMalloc and the device-wide
   synchronization it may bring.  Scratch comes from one fixed 8 MiB array
   per GPU, held by every GPU that loads the library until the process exits;
   products whose scratch does not fit (transform lengths above 2^19 for a
   square or 2^18 for two distinct operands, about 130 000 and 65 000 limbs
   per operand), or that need the split multiply, return FFG_E_RANGE with the
   bytes needed in the message.  ffg_init must have run first: it builds the
   device tables, looks the array's address up (with the device current) and
   loads the kernels used here, so the first call allocates nothing either.
   All calls share the one array, and it keeps the last call's contents:
   calls whose GPU work overlaps (different streams, no ordering between
   them) race and corrupt each other's results. */
int ffg_mul_device_noalloc(uint64_t *out, const uint64_t *a, size_t na, uint64_t bits_a, const uint64_t *b,
                           size_t nb, uint64_t bits_b, int square, void *stream);

/* One product sharded over GPUs by prime (one process per GPU; no counterpart
   in the reference, whose three primes run on one host, src/mul_ntt.c:97-118).
   ffg_mul_residues runs the forward transforms, the pointwise product and the
   inverse of primes [prime0, prime0 + nprimes) only, for the plan
   ffg_plan_select gives (four-step plans only: FFG_E_RANGE for a one-CTA
   length or a split product).  y: 3 * plan.L words of device memory,
   prime-major; prime k's scaled convolution lands in y[k L .. k L + conv),
   the other primes' words are left as they are.  The caller exchanges the
   slices (an all-gather of 4 L bytes per prime), then ffg_crt_residues
   recombines all three primes of y into out (na + nb + 1 limbs of device
   memory, fully written), exactly the product ffg_mul_device writes.
   Arguments and stream as for ffg_mul_device. */
int ffg_mul_residues(uint32_t *y, const uint64_t *a, size_t na, uint64_t bits_a, const uint64_t *b, size_t nb,
                     uint64_t bits_b, int square, uint32_t prime0, uint32_t nprimes, void *stream);
int ffg_crt_residues(uint64_t *out, const uint32_t *y, size_t na, uint64_t bits_a, size_t nb, uint64_t bits_b,
                     int square, void *stream);

/* fibonacci (src/fib.c:211) from bit i0 down: continues fast doubling from
   the pair (F(k-1), F(k)), k = n >> i0, on the device and returns F(n) as a
   limb array in pinned host memory (free with ffg_free).  i0 >= 1. */
int ffg_fib_chain(uint64_t n, int i0, const uint64_t *fkm1, size_t nkm1, const uint64_t *fk, size_t nk,
                  uint64_t **out, size_t *nout);

/* Device timing of the last ffg_fib_chain call, in milliseconds (CUDA events
   around the chain on its stream; excludes the host prefix and copies). */
double ffg_last_chain_ms(void);
/* Bytes the last ffg_fib_chain copied host -> device and device -> host. */
void ffg_last_chain_io(uint64_t *h2d_bytes, uint64_t *d2h_bytes);

/* Selects the CUDA device for every later call (one process per GPU); call
   before the first other entry point. */
int ffg_set_device(int device);

/* Kernel-family profiling for the roofline: with profiling on, every launch
   of a family is bracketed by CUDA events on its own stream; read returns the
   launches, summed device milliseconds and summed algorithmic bytes since
   ffg_profile() was last called.  Families: 0 one-CTA convolution, 1 forward
   column pass, 2 row pass (forward, pointwise, inverse), 3 inverse column
   pass, 4 CRT, 5 carry settle, 6 linear pass, 7 schoolbook. */
void ffg_profile(uint32_t family_mask); /* bit k on: bracket family k; 0: off */
int ffg_profile_read(int kind, uint64_t *launches, double *ms, double *bytes);
/* Kernel launches made by the library since it was loaded. */
uint64_t ffg_launch_count(void);

const char *ffg_last_error(void);
/* Frees an array this layer returned (ffg_fib_chain's results live in a
   pool of pinned host buffers; anything else is plain malloc memory). */
void ffg_free(void *p);
/* Returns 1 and takes p back into the pool if it is one of this layer's
   pinned result buffers, else 0 (p untouched). */
int ffg_release(void *p);
/* Releases device memory, streams and tables. */
void ffg_shutdown(void);

#ifdef __cplusplus
}
#endif
#endif
