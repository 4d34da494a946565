// Carry propagation by function composition, for the CRT and the linear
// passes (fast-doubling step, last factors).
//
// A kernel cuts its output into chunks of limbs and computes each chunk with
// carry-in 0, giving the chunk's limbs `low` and carry-out `out`.  A real
// carry-in c (signed, |c| < 2^100) changes the carry-out to
//     out + floor((low + c) / 2^(64 k))  in  {out - 1, out, out + 1},
// +1 only if limbs 2.. are all ones and c >= 2^128 - low01, -1 only if limbs
// 2.. are all zero and c < -low01 (low01 = the lowest 128 bits).  So every
// chunk's map c_in -> c_out is a step function with at most three values,
// and so is any composition of them: (tlo, thi, va, vb, vc).  The chunks'
// maps are scanned inside the CTA (warp shuffles + shared memory), the CTAs'
// maps by one warp, and a last pass adds each chunk's carry-in to its lowest
// limbs (rippling only through all-ones / all-zero limbs).  No kernel waits
// on another CTA, so nothing can spin.
//
// The reference does the same job with sequential chunks and a serial
// fix-up of their carries (src/crt.c:156-194, src/fib.c:81-109).
#pragma once
#include "ffg_internal.h"

namespace ffg {

typedef __int128 i128;
typedef unsigned __int128 u128;

FFG_DEV_INLINE i128 i128_max() { return (i128)(((u128)1 << 127) - 1); }
FFG_DEV_INLINE i128 i128_min() { return -i128_max() - 1; }

// The map of one chunk from its carry-out, low 128 bits and limb flags.
FFG_DEV_INLINE StepFn chunk_fn(i128 out, u128 low01, bool upper_ones, bool upper_zero) {
    const u128 LIM = (u128)1 << 100;
    StepFn f;
    f.va = out - 1;
    f.vb = out;
    f.vc = out + 1;
    f.tlo = i128_min();
    f.thi = i128_max();
    if (upper_ones) {
        u128 d = (u128)0 - low01;
        if (low01 != 0 && d < LIM) f.thi = (i128)d;
    }
    if (upper_zero && low01 < LIM) f.tlo = -(i128)low01;
    return f;
}

FFG_DEV_INLINE StepFn const_fn(i128 v) {
    StepFn f;
    f.tlo = i128_min();
    f.thi = i128_max();
    f.va = f.vb = f.vc = v;
    return f;
}

FFG_DEV_INLINE i128 fn_apply(const StepFn &f, i128 c) { return c < f.tlo ? f.va : (c >= f.thi ? f.vc : f.vb); }

// g after f (f is applied first).
FFG_DEV_INLINE StepFn fn_then(const StepFn &f, const StepFn &g) {
    StepFn r;
    r.tlo = f.tlo;
    r.thi = f.thi;
    r.va = fn_apply(g, f.va);
    r.vb = fn_apply(g, f.vb);
    r.vc = fn_apply(g, f.vc);
    return r;
}

FFG_DEV_INLINE i128 shfl_up_i128(i128 v, int d) {
    uint64_t lo = (uint64_t)v, hi = (uint64_t)((u128)v >> 64);
    lo = __shfl_up_sync(0xffffffffu, lo, d);
    hi = __shfl_up_sync(0xffffffffu, hi, d);
    return (i128)(((u128)hi << 64) | lo);
}

FFG_DEV_INLINE StepFn shfl_up_fn(const StepFn &f, int d) {
    StepFn r;
    r.tlo = shfl_up_i128(f.tlo, d);
    r.thi = shfl_up_i128(f.thi, d);
    r.va = shfl_up_i128(f.va, d);
    r.vb = shfl_up_i128(f.vb, d);
    r.vc = shfl_up_i128(f.vc, d);
    return r;
}

// Inclusive scan of one map per thread over the CTA (blockDim.x a multiple of
// 32, at most 1024): returns f_t o ... o f_0.  `warp_tot` is scratch of
// blockDim.x / 32 entries.
FFG_DEV_INLINE StepFn cta_scan(StepFn f, StepFn *warp_tot) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        StepFn g = shfl_up_fn(f, d);
        if (lane >= d) f = fn_then(g, f);
    }
    if (lane == 31) warp_tot[warp] = f;
    __syncthreads();
    if (warp > 0) {
        StepFn pre = warp_tot[0];
        for (int w = 1; w < warp; w++) pre = fn_then(pre, warp_tot[w]);
        f = fn_then(pre, f);
    }
    (void)nw;
    __syncthreads();
    return f;
}

// Adds the signed c into limbs d[0..n) (n >= 2) in place, rippling the carry
// or borrow out of the lowest 128 bits upward while it lasts; what leaves
// limb n-1 is accounted for by the next chunk's carry-in.
FFG_DEV_INLINE void add_carry_in(uint64_t *d, uint64_t n, i128 c) {
    if (c == 0 || n == 0) return;
    if (n == 1) {
        d[0] += (uint64_t)c;
        return;
    }
    u128 low = ((u128)d[1] << 64) | d[0];
    u128 s = low + (u128)c;
    d[0] = (uint64_t)s;
    d[1] = (uint64_t)(s >> 64);
    if (c > 0) {
        if (s >= low) return;            // no carry out of 128 bits
        for (uint64_t i = 2; i < n; i++)
            if (++d[i] != 0) return;
    } else {
        if (s <= low) return;            // no borrow out of 128 bits
        for (uint64_t i = 2; i < n; i++)
            if (d[i]-- != 0) return;
    }
}

} // namespace ffg
