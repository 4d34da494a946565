/*
 * Host side of the reference's Big surface: allocation with the reference's
 * out-of-memory behaviour, and the linear-time limb arithmetic the dispatch,
 * Toom-3 and the decimal conversion use (src/bigint.c, src/alloc.c).
 * Written for this layer; the products past the thresholds go to the GPU.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "fastfib.h"
#include "ffg.h"
#include "host_internal.h"

/* The reference ends the program with a message when memory runs out
   (src/alloc.c:143-146); so does this layer. */
void ff_out_of_memory(size_t bytes) {
    fprintf(stderr, "fastfib: out of memory (%zu bytes)\n", bytes);
    exit(1);
}

void ff_gpu_failed(const char *what, const char *msg) {
    fprintf(stderr, "fastfib: GPU %s failed: %s\n", what, msg);
    exit(1);
}

void *xmalloc(size_t bytes) {
    void *p = malloc(bytes ? bytes : 8);
    if (!p) ff_out_of_memory(bytes);
    return p;
}

void *xcalloc(size_t n, size_t size) {
    void *p = calloc(n ? n : 1, size ? size : 1);
    if (!p) ff_out_of_memory(n * size);
    return p;
}

/* Results of the device chain live in the layer's pinned buffers; everything
   else is the C heap. */
void xfree(void *p) {
    if (!ffg_release(p)) free(p);
}

/* The shared zero of empty views: never written, never freed (src/common.h:38-40). */
uint64_t g_zero_limb = 0;

double plat_seconds(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

size_t normalize_len(const uint64_t *d, size_t n) {
    while (n > 1 && d[n - 1] == 0) n--;
    return n;
}

void big_free(Big *x) {
    if (x->d != &g_zero_limb) xfree(x->d);
    x->d = NULL;
    x->n = 0;
}

Big big_from_u64(uint64_t v) {
    Big r = {xmalloc(sizeof(uint64_t)), 1};
    r.d[0] = v;
    return r;
}

int big_is_zero(const Big *a) { return a->n == 1 && a->d[0] == 0; }

size_t big_bits(const Big *a) { return 64 * (a->n - 1) + (64 - (size_t)__builtin_clzll(a->d[a->n - 1])); }

Big view_slice(const Big *a, size_t lo, size_t hi) {
    if (hi > a->n) hi = a->n;
    if (lo >= hi) return (Big){&g_zero_limb, 1};
    return (Big){a->d + lo, normalize_len(a->d + lo, hi - lo)};
}

Big big_copy(const Big *a) {
    Big r = {xmalloc(a->n * sizeof(uint64_t)), a->n};
    memcpy(r.d, a->d, a->n * sizeof(uint64_t));
    return r;
}

int big_cmp(const Big *a, const Big *b) {
    if (a->n != b->n) return a->n < b->n ? -1 : 1;
    for (size_t i = a->n; i-- > 0;)
        if (a->d[i] != b->d[i]) return a->d[i] < b->d[i] ? -1 : 1;
    return 0;
}

typedef unsigned __int128 u128;

/* x + y + c (c in {0, 1}) into *out; returns the carry out. */
static inline unsigned adc(uint64_t x, uint64_t y, unsigned c, uint64_t *out) {
    u128 s = (u128)x + y + c;
    *out = (uint64_t)s;
    return (unsigned)(s >> 64);
}

/* x - y - b (b in {0, 1}) into *out; returns the borrow out. */
static inline unsigned sbb(uint64_t x, uint64_t y, unsigned b, uint64_t *out) {
    u128 s = (u128)x - y - b;
    *out = (uint64_t)s;
    return (unsigned)(s >> 64) & 1;
}

/* Adds v at limb pos and ripples; returns the carry out of d[len-1]. */
uint64_t ff_ripple_add(uint64_t *d, size_t len, size_t pos, uint64_t v) {
    for (; v && pos < len; pos++) {
        d[pos] += v;
        v = d[pos] < v;
    }
    return v;
}

uint64_t ff_ripple_sub(uint64_t *d, size_t len, size_t pos, uint64_t v) {
    for (; v && pos < len; pos++) {
        uint64_t old = d[pos];
        d[pos] = old - v;
        v = old < v;
    }
    return v;
}

Big big_add(const Big *a, const Big *b) {
    if (a->n < b->n) {
        const Big *t = a;
        a = b;
        b = t;
    }
    size_t n = a->n + 1;
    uint64_t *d = xmalloc(n * sizeof(uint64_t));
    unsigned c = 0;
    for (size_t i = 0; i < b->n; i++) c = adc(a->d[i], b->d[i], c, &d[i]);
    memcpy(d + b->n, a->d + b->n, (a->n - b->n) * sizeof(uint64_t));
    d[a->n] = 0;
    ff_ripple_add(d, n, b->n, c);
    return (Big){d, normalize_len(d, n)};
}

Big big_sub(const Big *a, const Big *b) {
    size_t bn = b->n < a->n ? b->n : a->n;
    uint64_t *d = xmalloc(a->n * sizeof(uint64_t));
    unsigned c = 0;
    for (size_t i = 0; i < bn; i++) c = sbb(a->d[i], b->d[i], c, &d[i]);
    memcpy(d + bn, a->d + bn, (a->n - bn) * sizeof(uint64_t));
    ff_ripple_sub(d, a->n, bn, c);
    return (Big){d, normalize_len(d, a->n)};
}

uint64_t big_add_at(uint64_t *d, size_t dn, const Big *x, size_t off) {
    if (big_is_zero(x)) return 0;
    size_t xn = normalize_len(x->d, x->n);
    unsigned c = 0;
    for (size_t i = 0; i < xn; i++) c = adc(d[off + i], x->d[i], c, &d[off + i]);
    return ff_ripple_add(d, dn, off + xn, c);
}

void big_sub_at(uint64_t *d, size_t dn, const Big *x, size_t off) {
    if (big_is_zero(x)) return;
    size_t xn = normalize_len(x->d, x->n);
    unsigned c = 0;
    for (size_t i = 0; i < xn; i++) c = sbb(d[off + i], x->d[i], c, &d[off + i]);
    ff_ripple_sub(d, dn, off + xn, c);
}

void big_sub_inplace(Big *x, const Big *y) {
    big_sub_at(x->d, x->n, y, 0);
    x->n = normalize_len(x->d, x->n);
}

void big_add_inplace(Big *x, const Big *y) {
    if (y->n > x->n || x->d == &g_zero_limb) {
        Big t = big_add(x, y);
        big_free(x);
        *x = t;
        return;
    }
    if (big_add_at(x->d, x->n, y, 0)) {
        size_t n = x->n;
        uint64_t *d = xmalloc((n + 1) * sizeof(uint64_t));
        memcpy(d, x->d, n * sizeof(uint64_t));
        d[n] = 1;
        big_free(x);
        x->d = d;
        x->n = n + 1;
    }
}

void big_add_u64_inplace(Big *x, uint64_t v) {
    Big t = {&v, 1};
    big_add_inplace(x, &t);
}

void big_sub_u64_inplace(Big *x, uint64_t v) {
    Big t = {&v, 1};
    big_sub_inplace(x, &t);
}

Big big_shl1(const Big *a) { return big_shl_bits(a, 1); }

Big big_shr_bits(const Big *a, size_t k) {
    size_t s = k / 64, b = k % 64;
    if (s >= a->n) return big_from_u64(0);
    size_t n = a->n - s;
    uint64_t *d = xmalloc(n * sizeof(uint64_t));
    for (size_t i = 0; i < n; i++) {
        uint64_t lo = a->d[i + s], hi = i + s + 1 < a->n ? a->d[i + s + 1] : 0;
        d[i] = b ? (lo >> b) | (hi << (64 - b)) : lo;
    }
    return (Big){d, normalize_len(d, n)};
}

Big big_shl_bits(const Big *a, size_t k) {
    if (big_is_zero(a)) return big_from_u64(0);
    size_t s = k / 64, b = k % 64, n = a->n + s + 1;
    uint64_t *d = xcalloc(n, sizeof(uint64_t)), prev = 0;
    for (size_t i = 0; i < a->n; i++) {
        d[i + s] = b ? (a->d[i] << b) | (prev >> (64 - b)) : a->d[i];
        prev = a->d[i];
    }
    d[n - 1] = b ? prev >> (64 - b) : 0;
    return (Big){d, normalize_len(d, n)};
}

Big big_pow2(size_t k) {
    Big r = {xcalloc(k / 64 + 1, sizeof(uint64_t)), k / 64 + 1};
    r.d[k / 64] = 1ull << (k % 64);
    return r;
}

Big big_mul_schoolbook(const Big *a, const Big *b) {
    if (big_is_zero(a) || big_is_zero(b)) return big_from_u64(0);
    size_t n = a->n + b->n;
    uint64_t *d = xcalloc(n, sizeof(uint64_t));
    for (size_t i = 0; i < a->n; i++) {
        uint64_t ai = a->d[i], c = 0;
        if (!ai) continue;
        for (size_t j = 0; j < b->n; j++) {
            u128 t = (u128)ai * b->d[j] + d[i + j] + c;
            d[i + j] = (uint64_t)t;
            c = (uint64_t)(t >> 64);
        }
        d[i + b->n] = c;
    }
    return (Big){d, normalize_len(d, n)};
}

/* Cross products once, doubled, plus the squares (src/bigint.c:282-320). */
Big big_sqr_schoolbook(const Big *a) {
    if (big_is_zero(a)) return big_from_u64(0);
    size_t n = a->n, cap = 2 * n + 1;
    uint64_t *d = xcalloc(cap, sizeof(uint64_t));
    for (size_t i = 0; i < n; i++) {
        uint64_t ai = a->d[i], c = 0;
        if (!ai) continue;
        for (size_t j = i + 1; j < n; j++) {
            u128 t = (u128)ai * a->d[j] + d[i + j] + c;
            d[i + j] = (uint64_t)t;
            c = (uint64_t)(t >> 64);
        }
        d[i + n] = c;
    }
    uint64_t top = 0, c = 0;
    for (size_t i = 0; i < 2 * n; i++) { /* double */
        uint64_t v = d[i];
        d[i] = (v << 1) | top;
        top = v >> 63;
    }
    for (size_t i = 0; i < n; i++) { /* add the squares a[i]^2 at 2i */
        u128 sq = (u128)a->d[i] * a->d[i];
        u128 t = (u128)d[2 * i] + (uint64_t)sq + c;
        d[2 * i] = (uint64_t)t;
        t = (u128)d[2 * i + 1] + (uint64_t)(sq >> 64) + (uint64_t)(t >> 64);
        d[2 * i + 1] = (uint64_t)t;
        c = (uint64_t)(t >> 64);
    }
    d[2 * n] = top + c;
    return (Big){d, normalize_len(d, cap)};
}
