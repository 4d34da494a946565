/*
 * big_to_string (src/decimal.c:229-281): the decimal digits of a Big in a
 * malloc'd, NUL-terminated string the caller frees.
 *
 * Numbers of DEC_DEVICE_BITS bits and more convert on the GPU
 * (ffg_to_decimal_host: divide and conquer over 10^(19 2^l), every level's
 * Barrett products batched).  Smaller ones -- at most 4933 digits -- convert
 * here by Horner's rule in base 10^9: every 32-bit half of the number, top
 * first, enters as c <- c 2^32 + h over the base-10^9 chunks of c.  A chunk
 * times 2^32 plus the incoming carry stays below 2^63, so the whole loop runs
 * in 64-bit arithmetic with division by a constant; at this size its
 * quadratic cost is a few hundred thousand such steps.
 */
#include <stdlib.h>
#include <string.h>

#include "fastfib.h"
#include "ffg.h"
#include "host_internal.h"

/* Numbers of at least this many bits convert on the device; the device path
   takes every number above 10^2432 (about 8080 bits), so both sides of the
   boundary are covered. */
#define DEC_DEVICE_BITS 16384
#define DEC_CHUNK 1000000000u /* 10^9 */

static char *small_to_string(const Big *a) {
    const size_t halves = 2 * a->n;
    /* decimal digits <= bits log10(2) + 1 < 32 halves 0.30103 + 1 */
    const size_t cap = (halves * 32 * 30103 / 100000 + 1) / 9 + 2;
    uint32_t *c = xcalloc(cap, sizeof(uint32_t));
    size_t m = 0; /* chunks in use, little-endian */
    for (size_t k = halves; k-- > 0;) {
        uint64_t carry = (uint32_t)(a->d[k / 2] >> (32 * (k & 1)));
        for (size_t i = 0; i < m; i++) {
            const uint64_t t = ((uint64_t)c[i] << 32) + carry;
            c[i] = (uint32_t)(t % DEC_CHUNK);
            carry = t / DEC_CHUNK;
        }
        while (carry) {
            c[m++] = (uint32_t)(carry % DEC_CHUNK);
            carry /= DEC_CHUNK;
        }
    }
    char *s = malloc(9 * (m ? m : 1) + 1);
    if (!s) ff_out_of_memory(9 * (m ? m : 1) + 1);
    size_t n = 0;
    if (m == 0) {
        s[n++] = '0';
    } else {
        char top[10];
        int t = 0;
        for (uint32_t v = c[m - 1]; v; v /= 10) top[t++] = (char)('0' + v % 10);
        while (t) s[n++] = top[--t];
        for (size_t i = m - 1; i-- > 0;) {
            uint32_t v = c[i];
            for (int j = 8; j >= 0; j--, v /= 10) s[n + (size_t)j] = (char)('0' + v % 10);
            n += 9;
        }
    }
    s[n] = 0;
    xfree(c);
    return s;
}

char *big_to_string(const Big *a) {
    if (big_is_zero(a) || big_bits(a) < DEC_DEVICE_BITS) return small_to_string(a);
    char *s = NULL;
    size_t n = 0;
    int done = 0;
    if (ffg_to_decimal_host(a->d, a->n, &s, &n, &done)) ff_gpu_failed("decimal conversion", ffg_last_error());
    /* the device path declines only numbers below 10^2432, or on an estimate
       its bounds rule out: either is a fault here, reported like a GPU failure */
    if (!done) ff_gpu_failed("decimal conversion", ffg_last_error());
    char *m = xmalloc(n + 1); /* big_to_string's result is the caller's to free() */
    memcpy(m, s, n + 1);
    ffg_free(s);
    return m;
}
