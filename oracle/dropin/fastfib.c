/*
 * Drop-in check (test infrastructure, not product code).
 *
 * The reference's test harnesses (tests/hexfib.c, nttfuzz.c, bound.c,
 * dectest.c) compile the whole reference into themselves with
 * `#include "../fastfib.c"` (tests/hexfib.c:3-4).  `make -C oracle dropin`
 * compiles each harness, unmodified, with this file standing in that place:
 * it brings in the library's C surface (include/fastfib.h: Big, big_mul,
 * big_mul_ntt, fibonacci, big_to_string, ntt_init, g_ntt_max_L and the
 * helpers the harnesses call) and the headers the reference's amalgamation
 * would have pulled in, and the harness links against libfastfib_b200.so.
 * Nothing the harnesses expect to be static is defined here: every call goes
 * to the library.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "fastfib.h"

typedef unsigned __int128 u128; /* the reference's src/common.h:36 type */
