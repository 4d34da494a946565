/*
 * fibonacci(n) by fast doubling (src/fib.c:211-261): walk the bits of n from
 * the top keeping (F(k-1), F(k)); each bit costs two squarings and one linear
 * pass, the last bit one multiply:
 *     F(2k-1) = F(k)^2 + F(k-1)^2
 *     F(2k+1) = 4 F(k)^2 - F(k-1)^2 + 2(-1)^k
 *     F(2k)   = F(2k+1) - F(2k-1)
 *     F(2k)   = F(k) (F(k) + 2 F(k-1)),  F(2k+1) = (2F(k) + F(k-1)) (2F(k) - F(k-1)) + 2(-1)^k
 * The short prefix (operands below FIB_GPU_START_LIMBS) runs here on the
 * host; from there the chain stays on the device (ffg_fib_chain) until the
 * result is copied back.
 */
#include "fastfib.h"
#include "ffg.h"
#include "host_internal.h"

#ifndef FIB_GPU_START_LIMBS
#define FIB_GPU_START_LIMBS 48
#endif

#define LOG2_PHI 0.6942419136306174

/* A = s1 + s2, B = 4 s1 - s2 + 2(-1)^k, C = B - A; keeps (C, B) if bit else (A, C). */
static void step_linear(const Big *s1, const Big *s2, int k_odd, int bit, Big *lo, Big *hi) {
    Big A = big_add(s1, s2);
    Big s4 = big_shl_bits(s1, 2);
    Big B = big_sub(&s4, s2);
    big_free(&s4);
    if (k_odd) big_sub_u64_inplace(&B, 2);
    else big_add_u64_inplace(&B, 2);
    Big C = big_sub(&B, &A);
    if (bit) {
        *lo = C;
        *hi = B;
        big_free(&A);
    } else {
        *lo = A;
        *hi = C;
        big_free(&B);
    }
}

Big fibonacci(uint64_t n) {
    if (n == 0) return big_from_u64(0);
    ntt_init((size_t)((double)n * LOG2_PHI / 64.0) + 8);
    Big fkm1 = big_from_u64(0), fk = big_from_u64(1);
    int k_odd = 1, top = 63 - __builtin_clzll(n);
    int i = top - 1;
    for (; i >= 1 && fk.n < FIB_GPU_START_LIMBS; i--) {
        Big s1 = big_sqr(&fk), s2 = big_sqr(&fkm1);
        big_free(&fkm1);
        big_free(&fk);
        int bit = (int)((n >> i) & 1);
        step_linear(&s1, &s2, k_odd, bit, &fkm1, &fk);
        big_free(&s1);
        big_free(&s2);
        k_odd = bit;
    }
    if (top == 0) {
        big_free(&fkm1);
        return fk;
    }
    if (i >= 0 && fk.n >= FIB_GPU_START_LIMBS) {
        /* the rest of the chain, the last bit included, on the device;
           bits top-1 .. i+1 are done, so k = n >> (i + 1) */
        uint64_t *d = NULL;
        size_t nd = 0;
        int rc = ffg_fib_chain(n, i + 1, fkm1.d, fkm1.n, fk.d, fk.n, &d, &nd);
        if (rc) ff_gpu_failed("fibonacci chain", ffg_last_error());
        big_free(&fkm1);
        big_free(&fk);
        return (Big){d, nd}; /* the layer's pinned buffer: big_free returns it */
    }
    /* short n: the last bit here as well */
    Big result;
    if (n & 1) {
        Big u2 = big_shl_bits(&fk, 1);
        Big x = big_add(&u2, &fkm1), y = big_sub(&u2, &fkm1);
        big_free(&u2);
        big_free(&fk);
        big_free(&fkm1);
        result = big_mul(&x, &y);
        big_free(&x);
        big_free(&y);
        if (k_odd) big_sub_u64_inplace(&result, 2);
        else big_add_u64_inplace(&result, 2);
    } else {
        Big v2 = big_shl_bits(&fkm1, 1);
        Big x = big_add(&fk, &v2);
        big_free(&v2);
        big_free(&fkm1);
        result = big_mul(&fk, &x);
        big_free(&x);
        big_free(&fk);
    }
    return result;
}
