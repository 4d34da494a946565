/*
 * big_to_string (src/decimal.c:229-281): divide and conquer over
 * P_i = 10^(19 2^i).  x < P_i^2 splits as q P_i + r by Barrett division with a
 * Newton reciprocal of P_i (two products, the NTT on the GPU once large), and
 * q and r become the two halves of its 2 * 19 * 2^i digits; pieces below
 * P_DEC_LEAF_LG^2 are converted by repeated division by 10^19.
 */
#include <stdlib.h>
#include <string.h>

#include "fastfib.h"
#include "ffg.h"
#include "host_internal.h"

#ifndef DEC_LEAF_LG
#define DEC_LEAF_LG 4
#endif
#define DEC_P0 10000000000000000000ull /* 10^19 */

typedef unsigned __int128 u128;

/* floor(2^(2s) / P) minus at most 4, for P of exactly s bits (src/decimal.c:39-71). */
static Big big_recip(const Big *P, size_t s) {
    if (s <= 62) return big_from_u64((uint64_t)(((u128)1 << (2 * s)) / P->d[0]));
    size_t h = (s + 1) / 2 + 16;
    Big Ph = big_shr_bits(P, s - h);
    Big mh = big_recip(&Ph, h);
    big_free(&Ph);
    Big y = big_shl_bits(&mh, s - h);
    big_free(&mh);
    Big Z = big_pow2(2 * s), d = big_mul(P, &y);
    int below = big_cmp(&d, &Z) <= 0;
    Big e = below ? big_sub(&Z, &d) : big_sub(&d, &Z);
    big_free(&d);
    Big ye = big_mul(&y, &e);
    big_free(&e);
    Big corr = big_shr_bits(&ye, 2 * s);
    big_free(&ye);
    if (below) big_add_inplace(&y, &corr);
    else big_sub_inplace(&y, &corr);
    big_free(&corr);
    big_free(&Z);
    big_sub_u64_inplace(&y, 2);
    return y;
}

/* q = floor(x / P), r = x mod P for x < 2^(2s) (src/decimal.c:76-89). */
static void divmod_barrett(const Big *x, const Big *P, const Big *m, size_t s, Big *q, Big *r) {
    Big q1 = big_shr_bits(x, s - 1);
    Big t = big_mul(&q1, m);
    big_free(&q1);
    *q = big_shr_bits(&t, s + 1);
    big_free(&t);
    Big qp = big_mul(q, P);
    *r = big_sub(x, &qp);
    big_free(&qp);
    while (big_cmp(r, P) >= 0) {
        big_sub_inplace(r, P);
        big_add_u64_inplace(q, 1);
    }
}

/* The unbalanced top split (src/decimal.c:95-125). */
static void divmod_any(const Big *x, const Big *P, size_t s, Big *q, Big *r) {
    size_t bx = big_is_zero(x) ? 0 : big_bits(x);
    if (bx < s) {
        *q = big_from_u64(0);
        *r = big_copy(x);
        return;
    }
    size_t t = bx - s + 1, k = t + 64 < s ? t + 64 : s;
    Big Pk = big_shr_bits(P, s - k), Xk = big_shr_bits(x, s - k);
    Big mk = big_recip(&Pk, k), rk;
    divmod_barrett(&Xk, &Pk, &mk, k, q, &rk);
    big_free(&Pk);
    big_free(&Xk);
    big_free(&mk);
    big_free(&rk);
    Big qp = big_mul(q, P);
    while (big_cmp(&qp, x) > 0) {
        big_sub_u64_inplace(q, 1);
        big_sub_inplace(&qp, P);
    }
    *r = big_sub(x, &qp);
    big_free(&qp);
    while (big_cmp(r, P) >= 0) {
        big_sub_inplace(r, P);
        big_add_u64_inplace(q, 1);
    }
}

/* Exactly 19 * chunks digits of x < 10^(19 chunks), zero padded (src/decimal.c:139-150). */
static void dec_leaf(const Big *x, size_t chunks, char *out) {
    size_t n = x->n;
    uint64_t *t = xmalloc(n * sizeof(uint64_t));
    memcpy(t, x->d, n * sizeof(uint64_t));
    for (size_t c = chunks; c-- > 0;) {
        uint64_t rem = 0;
        for (size_t i = n; i-- > 0;) {
            u128 cur = ((u128)rem << 64) | t[i];
            t[i] = (uint64_t)(cur / DEC_P0);
            rem = (uint64_t)(cur % DEC_P0);
        }
        while (n > 1 && t[n - 1] == 0) n--;
        char *o = out + 19 * c;
        for (int j = 18; j >= 0; j--, rem /= 10) o[j] = (char)('0' + rem % 10);
    }
    xfree(t);
}

typedef struct {
    Big pw[48], inv[48];
    size_t bits[48];
} DecCtx;

static void dec_emit(const DecCtx *c, Big x, int lvl, char *out) {
    if (lvl <= DEC_LEAF_LG) {
        dec_leaf(&x, (size_t)2 << lvl, out);
        big_free(&x);
        return;
    }
    Big q, r;
    divmod_barrett(&x, &c->pw[lvl], &c->inv[lvl], c->bits[lvl], &q, &r);
    big_free(&x);
    dec_emit(c, q, lvl - 1, out);
    dec_emit(c, r, lvl - 1, out + ((size_t)19 << lvl));
}

/* Numbers of at least this many bits convert on the device (ffg_to_decimal_host:
   every level's Barrett products batched); smaller ones here. */
#define DEC_DEVICE_BITS 16384

char *big_to_string(const Big *a) {
    if (big_is_zero(a)) {
        char *s = malloc(2);
        if (!s) ff_out_of_memory(2);
        s[0] = '0';
        s[1] = 0;
        return s;
    }
    if (big_bits(a) >= DEC_DEVICE_BITS) {
        char *s = NULL;
        size_t n = 0;
        int done = 0;
        if (ffg_to_decimal_host(a->d, a->n, &s, &n, &done)) ff_gpu_failed("decimal conversion", ffg_last_error());
        if (done) { /* big_to_string's result is the caller's to free() */
            char *m = xmalloc(n + 1);
            memcpy(m, s, n + 1);
            ffg_free(s);
            return m;
        }
        /* declined (a correction out of range): the level-by-level path below */
    }
    DecCtx *c = xmalloc(sizeof(DecCtx));
    size_t ba = big_bits(a);
    int T = 0;
    c->pw[0] = big_from_u64(DEC_P0);
    c->bits[0] = big_bits(&c->pw[0]);
    while (2 * (c->bits[T] - 1) < ba) {
        c->pw[T + 1] = big_sqr(&c->pw[T]);
        c->bits[T + 1] = big_bits(&c->pw[T + 1]);
        T++;
    }
    for (int i = DEC_LEAF_LG + 1; i < T; i++) c->inv[i] = big_recip(&c->pw[i], c->bits[i]);
    size_t half = (size_t)19 << T, total = 2 * half;
    char *buf = malloc(total + 1);
    if (!buf) ff_out_of_memory(total + 1);
    if (T <= DEC_LEAF_LG) {
        dec_leaf(a, (size_t)2 << T, buf);
    } else {
        Big q, r;
        divmod_any(a, &c->pw[T], c->bits[T], &q, &r);
        dec_emit(c, q, T - 1, buf);
        dec_emit(c, r, T - 1, buf + half);
    }
    for (int i = 0; i <= T; i++) big_free(&c->pw[i]);
    for (int i = DEC_LEAF_LG + 1; i < T; i++) big_free(&c->inv[i]);
    xfree(c);
    size_t z = 0;
    while (z + 1 < total && buf[z] == '0') z++;
    memmove(buf, buf + z, total - z);
    buf[total - z] = 0;
    return buf;
}
