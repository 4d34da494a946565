/*
 * fastfib.h -- the reference's C surface, served by the B200 layer.
 *
 * Same names, argument meaning, ownership and error behaviour as the
 * reference's unity build (shwwwa/fastfib), so its callers and test harnesses
 * keep working; behind big_mul_ntt, fibonacci and big_to_string the work runs
 * on the GPU through include/ffg.h.
 *
 *   Big                 src/common.h:29-33   little-endian 64-bit limbs, normalized
 *   big_mul / big_sqr   src/mul_basic.c:64,109   the threshold dispatch
 *   big_mul_ntt         src/mul_ntt.c:97     the NTT multiply (square: a == b)
 *   ntt_init            src/ntt_tables.c:72  transform cap for max_limbs
 *   g_ntt_max_L         src/mul_basic.c:26   the cap itself (tests set it to 0)
 *   fibonacci           src/fib.c:211        F(n) by fast doubling
 *   big_to_string       src/decimal.c:229    decimal digits, caller frees (free)
 *
 * Ownership: every returned Big is new; free it with big_free.  Inputs are
 * never written or freed and may be views (view_slice).  Out of memory prints
 * a message and exits with status 1, as the reference's allocator does
 * (src/alloc.c:143-146); a GPU failure does the same with the layer's message.
 */
#ifndef FASTFIB_H
#define FASTFIB_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    uint64_t *d; /* limbs, lowest first */
    size_t n;    /* limbs; >= 1, no leading zero limb, zero is {0} */
} Big;

extern size_t g_ntt_max_L;

void *xmalloc(size_t bytes);
void *xcalloc(size_t n, size_t size);
void xfree(void *p);

size_t normalize_len(const uint64_t *d, size_t n);
void big_free(Big *x);
Big big_from_u64(uint64_t v);
int big_is_zero(const Big *a);
size_t big_bits(const Big *a);
Big view_slice(const Big *a, size_t lo, size_t hi);
Big big_copy(const Big *a);
int big_cmp(const Big *a, const Big *b);
Big big_add(const Big *a, const Big *b);
Big big_sub(const Big *a, const Big *b);
uint64_t big_add_at(uint64_t *d, size_t dn, const Big *x, size_t off);
void big_sub_at(uint64_t *d, size_t dn, const Big *x, size_t off);
void big_add_inplace(Big *x, const Big *y);
void big_sub_inplace(Big *x, const Big *y);
void big_add_u64_inplace(Big *x, uint64_t v);
void big_sub_u64_inplace(Big *x, uint64_t v);
Big big_shl1(const Big *a);
Big big_shr_bits(const Big *a, size_t k);
Big big_shl_bits(const Big *a, size_t k);
Big big_pow2(size_t k);
Big big_mul_schoolbook(const Big *a, const Big *b);
Big big_sqr_schoolbook(const Big *a);

void ntt_init(size_t max_limbs);
/* The run-time counterpart of the reference's -DNTT_MAX_LG (default 25). */
int ff_set_max_lg(int lg);
Big big_mul(const Big *a, const Big *b);
Big big_sqr(const Big *a);
Big big_mul_ntt(const Big *a, const Big *b);
Big big_mul_toom3(const Big *a, const Big *b);

Big fibonacci(uint64_t n);
char *big_to_string(const Big *a);
double plat_seconds(void);

#ifdef __cplusplus
}
#endif
#endif
