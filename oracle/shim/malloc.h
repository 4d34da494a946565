/*
 * Test-harness shim, NOT product code: the MSVC aligned-allocation pair the
 * reference's platform layer calls (src/platform_win.h:50-57), on POSIX.
 */
#ifndef FASTFIB_ORACLE_MALLOC_SHIM_H
#define FASTFIB_ORACLE_MALLOC_SHIM_H
#include <stdlib.h>

static inline void *_aligned_malloc(size_t bytes, size_t align) {
    void *p = NULL;
    if (align < sizeof(void *)) align = sizeof(void *);
    return posix_memalign(&p, align, bytes ? bytes : 1) == 0 ? p : NULL;
}
static inline void _aligned_free(void *p) { free(p); }

#endif
