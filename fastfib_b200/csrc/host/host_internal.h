/* Internal helpers shared by the host C files of the Big surface. */
#ifndef FF_HOST_INTERNAL_H
#define FF_HOST_INTERNAL_H
#include <stddef.h>
#include <stdint.h>

#include "fastfib.h"

extern uint64_t g_zero_limb;

void ff_out_of_memory(size_t bytes);
void ff_gpu_failed(const char *what, const char *msg);
uint64_t ff_ripple_add(uint64_t *d, size_t len, size_t pos, uint64_t v);
uint64_t ff_ripple_sub(uint64_t *d, size_t len, size_t pos, uint64_t v);

/* Sign + magnitude, for Toom-3's negative evaluation points (src/bigint.c:353-407). */
typedef struct {
    int neg;
    Big mag;
} SBig;

#endif
