/*
 * fastfib oracle: a plain, scalar C restatement of the reference's multiply
 * hot path, used ONLY as the checker by tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg.  Nothing in the product links or calls it.
 *
 * Parity pin: tests/test_oracle.py checks this restatement against the
 * reference's own known answers (tests/check.py's n list via fibonacci.py,
 * tests/bound.c's closed forms, tests/nttfuzz.c's generator, the fingerprints
 * of tests/fingerprint.py) and against the unmodified reference built from
 * its sources into oracle/_ref/ (oracle/Makefile).
 *
 * Numbers are little-endian arrays of 64-bit limbs.  Every returned array or
 * string is malloc'ed; free it with fo_free.
 */
#ifndef FASTFIB_ORACLE_H
#define FASTFIB_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* The choice big_mul_ntt makes for a product (src/mul_ntt.c:97-118), or the
   split's choice (src/mul_split.c:149-177) when split != 0. */
typedef struct {
    uint32_t width;   /* coefficient bits b */
    uint32_t lg;      /* L = 2^lg, or 3 * 2^lg when r3 */
    uint32_t r3;
    uint32_t split;   /* 1: the piecewise split multiply */
    uint64_t L;       /* transform length (split: the piece length Lp) */
    uint64_t conv;    /* coefficients of the product: ca + cb - 1 */
    uint64_t ca, cb;  /* coefficients of each operand */
    uint64_t ka, kb;  /* split only: pieces of each operand */
    uint64_t Lbig;    /* split only: (ka + kb) * Lp / 2 */
} FoPlan;

void fo_ntt_init(size_t max_limbs);
size_t fo_ntt_max_L(void);
void fo_set_ntt_max_L(size_t L);
void fo_set_max_lg(int lg); /* the reference's -DNTT_MAX_LG, at run time */
int fo_ntt_plan(uint64_t bits_a, uint64_t bits_b, int square, FoPlan *plan);

uint64_t *fo_mul(const uint64_t *a, size_t na, const uint64_t *b, size_t nb, int square, size_t *nout);
uint64_t *fo_mul_ntt(const uint64_t *a, size_t na, const uint64_t *b, size_t nb, int square, size_t *nout);
uint64_t *fo_mul_ntt_forced(const uint64_t *a, size_t na, const uint64_t *b, size_t nb, int square,
                            uint32_t width, uint64_t L, size_t *nout);
/* A product sharded by prime: prime k's scaled convolution at (width, L)
   into y[0 .. L) (-1 when L is too short); the product from all three
   primes' residues (3 L words). */
int fo_residues(const uint64_t *a, size_t na, const uint64_t *b, size_t nb, int square, uint32_t width,
                uint64_t L, int k, uint32_t *y);
uint64_t *fo_crt_residues(const uint32_t *y, uint64_t L, uint64_t conv, uint32_t width, size_t limbs,
                          size_t *nout);
uint64_t *fo_fibonacci(uint64_t n, size_t *nout);
char *fo_to_string(const uint64_t *a, size_t na);
void fo_fingerprint(const uint64_t *a, size_t na, uint64_t out[6]);
void fo_free(void *p);

/* The learned dispatch's cost model (mlp_oracle.c): parameter count, every
   output for n feature rows (n * 4 doubles), and the loss with its gradient
   (fo_mlp_nparam() doubles). */
size_t fo_mlp_nparam(void);
void fo_mlp_predict(const float *params, const float *X, size_t n, double *out);
double fo_mlp_grad(const float *params, const float *X, const int32_t *method, const float *y, size_t n,
                   double *grad);

#ifdef __cplusplus
}
#endif
#endif
