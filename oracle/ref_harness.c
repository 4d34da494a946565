/*
 * Test-harness only, NOT product code.  Compiles the UNMODIFIED reference
 * program (fastfib.c, a unity build whose functions are all static) into one
 * shared library and exports plain C wrappers around the functions the
 * parity tests and the CPU baseline need.  The reference's own test harnesses
 * reach its internals the same way: `#define UNIT_TEST_NO_MAIN` and
 * `#include "../fastfib.c"` (tests/hexfib.c:3-4, tests/nttfuzz.c:7-8).
 *
 * Only tests/, smoke() and bench.py's CPU-baseline / reference legs load the
 * library this file builds (oracle/_ref/libfastfib_ref.so).
 *
 * Every returned limb array or string is malloc'ed; free it with ffref_free.
 */
#define UNIT_TEST_NO_MAIN
#include "fastfib.c"

/* A read-only Big over caller limbs, normalized as Big requires
   (src/common.h:29-33): n >= 1, no leading zero limb, zero is {0}. */
static Big ffref_view(const uint64_t *d, size_t n) {
    if (n == 0 || d == NULL) return (Big){&g_zero_limb, 1};
    n = normalize_len(d, n);
    return (Big){(uint64_t *)d, n};
}

/* Copies r's limbs to a malloc'ed array, frees r, stores the limb count. */
static uint64_t *ffref_take(Big *r, size_t *nout) {
    uint64_t *o = (uint64_t *)malloc(r->n * sizeof(uint64_t));
    if (o) memcpy(o, r->d, r->n * sizeof(uint64_t));
    *nout = r->n;
    big_free(r);
    return o;
}

/** ntt_init (src/ntt_tables.c:72): root tables for products up to max_limbs. */
void ffref_ntt_init(size_t max_limbs) { ntt_init(max_limbs); }

/** The longest transform the tables allow right now (src/mul_basic.c:26). */
size_t ffref_ntt_max_L(void) { return g_ntt_max_L; }

/** Overrides g_ntt_max_L the way tests/nttfuzz.c:33-39 does (0 hides the NTT). */
void ffref_set_ntt_max_L(size_t L) { g_ntt_max_L = L; }

/** big_mul / big_sqr (src/mul_basic.c:64-132): the threshold dispatch. */
uint64_t *ffref_mul(const uint64_t *a, size_t na, const uint64_t *b, size_t nb, int square, size_t *nout) {
    Big A = ffref_view(a, na), B = ffref_view(b, nb);
    Big r = square ? big_sqr(&A) : big_mul(&A, &B);
    return ffref_take(&r, nout);
}

/** big_mul_ntt (src/mul_ntt.c:97): the NTT multiply; square signalled by a == b. */
uint64_t *ffref_mul_ntt(const uint64_t *a, size_t na, const uint64_t *b, size_t nb, int square, size_t *nout) {
    Big A = ffref_view(a, na), B = ffref_view(b, nb);
    Big r = big_mul_ntt(&A, square ? &A : &B);
    return ffref_take(&r, nout);
}

/** fibonacci (src/fib.c:211): F(n) by fast doubling. */
uint64_t *ffref_fibonacci(uint64_t n, size_t *nout) {
    Big r = fibonacci(n);
    return ffref_take(&r, nout);
}

/** big_to_string (src/decimal.c:229): decimal digits, no leading zeros. */
char *ffref_to_string(const uint64_t *a, size_t na) {
    Big A = ffref_view(a, na);
    return big_to_string(&A);
}

/** Frees an array or string returned above. */
void ffref_free(void *p) { free(p); }

/** The reference's monotonic clock (src/platform.h:38). */
double ffref_seconds(void) { return plat_seconds(); }

/** Logical CPUs the reference's pool uses (src/pool.c, plat_cpu_count). */
int ffref_cpus(void) { return plat_cpu_count(); }

/** The CPU baseline of the multiply microbench: `reps` calls of the
    reference's big_mul / big_sqr (its own threshold dispatch, NTT and thread
    pool, its NTT tables built first) on one operand pair, the results freed
    unread; returns the seconds of the fastest call, timed with the
    reference's clock. */
double ffref_time_mul(const uint64_t *a, size_t na, const uint64_t *b, size_t nb, int square, int reps) {
    Big A = ffref_view(a, na), B = ffref_view(b, nb);
    ntt_init(na + nb); /* tables first (untimed), as fibonacci() does */
    double best = 1e30;
    for (int i = 0; i < reps; i++) {
        double t = plat_seconds();
        Big r = square ? big_sqr(&A) : big_mul(&A, &B);
        t = plat_seconds() - t;
        big_free(&r);
        if (t < best) best = t;
    }
    return best;
}

/** The CPU baseline of a batch of independent products: products i < count
    of operands a + aoff[i] (na[i] limbs) and b + boff[i] (nb[i] limbs), one
    big_mul after another as the reference computes independent products
    (src/decimal.c:177-203 runs its products one at a time, each spread over
    the pool); returns the seconds for the whole batch. */
double ffref_time_mul_batch(const uint64_t *a, const size_t *aoff, const size_t *na, const uint64_t *b,
                            const size_t *boff, const size_t *nb, size_t count) {
    size_t most = 0;
    for (size_t i = 0; i < count; i++)
        if (na[i] + nb[i] > most) most = na[i] + nb[i];
    ntt_init(most); /* tables first (untimed) */
    double t = plat_seconds();
    for (size_t i = 0; i < count; i++) {
        Big A = ffref_view(a + aoff[i], na[i]), B = ffref_view(b + boff[i], nb[i]);
        Big r = big_mul(&A, &B);
        big_free(&r);
    }
    return plat_seconds() - t;
}
