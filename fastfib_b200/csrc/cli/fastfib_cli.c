/*
 * fastfib [n] [--print] [--help]: the reference's command line
 * (src/main.c:52-105) over this library's Big surface.  F(n) is computed by
 * fibonacci() (the chain on the GPU), and its wall time printed; --print
 * also converts it with big_to_string() and prints the digits and the
 * conversion time.  Arguments come in any order; n is one run of decimal
 * digits that fits 64 bits (no sign, no exponent, no hex: the reference's
 * parse_n, src/main.c:38-50), asked for on stdin when missing.  Bad input is
 * reported with exit status 1 before any GPU work starts.  The reference's
 * AVX2 start-up check (src/main.c:17-25) has no counterpart: a missing GPU is
 * reported by the library's first call, also with status 1.  For n large
 * enough to reach the GPU the device is set up before the timed call.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "fastfib.h"
#include "ffg.h"

static void print_usage(FILE *f) {
    fputs("usage: fastfib [n] [--print]\n"
          "  n        which Fibonacci number (asked for if missing)\n"
          "  --print  also print its decimal digits\n",
          f);
}

/* 1 and *out = the value when s is one or more decimal digits below 2^64. */
static int read_u64(const char *s, uint64_t *out) {
    if (*s == '\0') return 0;
    uint64_t v = 0;
    for (const char *p = s; *p; p++) {
        if (*p < '0' || *p > '9') return 0;
        const uint64_t d = (uint64_t)(*p - '0');
        if (v > UINT64_MAX / 10 || v * 10 > UINT64_MAX - d) return 0;
        v = v * 10 + d;
    }
    *out = v;
    return 1;
}

static double now_seconds(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

/* The streamed conversion's sink: one slice of digits to the output. */
static void write_digits(const char *d, size_t n, void *user) { fwrite(d, 1, n, (FILE *)user); }

int main(int argc, char **argv) {
    uint64_t n = 0;
    int got_n = 0, want_digits = 0;
    for (int i = 1; i < argc; i++) {
        const char *a = argv[i];
        if (!strcmp(a, "--help") || !strcmp(a, "-h")) {
            print_usage(stdout);
            return 0;
        }
        if (!strcmp(a, "--print")) {
            want_digits = 1;
            continue;
        }
        if (!got_n && read_u64(a, &n)) {
            got_n = 1;
            continue;
        }
        fprintf(stderr, "invalid argument: %s\n", a);
        print_usage(stderr);
        return 1;
    }
    if (!got_n) {
        char line[64];
        fputs("Enter n: ", stdout);
        fflush(stdout);
        if (!fgets(line, sizeof line, stdin)) return 1;
        char *s = line;
        if ((unsigned char)s[0] == 0xEF && (unsigned char)s[1] == 0xBB && (unsigned char)s[2] == 0xBF)
            s += 3; /* a UTF-8 byte order mark from piped input */
        while (*s == ' ' || *s == '\t') s++;
        size_t len = strcspn(s, " \t\r\n");
        s[len] = '\0';
        if (!read_u64(s, &n)) {
            fprintf(stderr, "invalid n: %s\n", s);
            return 1;
        }
    }

    /* numbers the GPU computes: the CUDA context, the kernels (loaded eagerly)
       and the tables are set up before the clock starts, so Time covers F(n) */
    if (n >= 4096) {
        setenv("CUDA_MODULE_LOADING", "EAGER", 0);
        if (ffg_init((size_t)((double)n * 0.6942419136306174 / 64.0) + 8)) {
            fprintf(stderr, "fastfib: GPU init failed: %s\n", ffg_last_error());
            return 1;
        }
    }

    double t0 = now_seconds();
    Big f = fibonacci(n);
    const double t_fib = now_seconds() - t0;

    double t_dec = 0;
    if (want_digits) {
        /* large numbers: the device conversion streams its digits out slice
           by slice, each slice written while the GPU works on the next;
           small ones (or a declined conversion, which emits nothing):
           big_to_string.  The time covers the conversion and the writes. */
        printf("fibonacci(%llu) = ", (unsigned long long)n);
        t0 = now_seconds();
        size_t nd = 0;
        int done = 0;
        if (f.n >= 256 && ffg_to_decimal_stream(f.d, f.n, write_digits, stdout, &nd, &done) != FFG_OK) {
            fprintf(stderr, "fastfib: decimal conversion failed: %s\n", ffg_last_error());
            return 1;
        }
        if (!done) {
            char *digits = big_to_string(&f);
            fputs(digits, stdout);
            free(digits);
        }
        t_dec = now_seconds() - t0;
        fputc('\n', stdout);
    }
    printf("Time: %.6f seconds\n", t_fib);
    if (want_digits) printf("Decimal conversion: %.6f seconds\n", t_dec);
    big_free(&f);
    return 0;
}
