// Limb sums and ripple carries, shared by the CRT and the linear passes.
//
// Both kernels first give every output limb j of their CTA a column sum
//     T_j = lo_j + 2^64 hi_j,   hi_j small and >= 0,
// (the CRT: the slices of the 3-4 coefficients X_i 2^(i b) that overlap limb
// j; the linear pass: alpha s1_j + beta s2_j with negative terms written in
// two's complement over the output length, so nothing is negative).  What is
// left is one addition, v_j = lo_j + hi_(j-1), whose carries are single bits:
// the carry into limb j+1 is g_j | (p_j & c_j) with g_j = (v_j overflowed) and
// p_j = (v_j == 2^64 - 1).  For 32 limbs held by a warp that chain is one
// 32-bit addition of ballots, A + B + c_in with A = G | P, B = G: bit k of
// (A + B + c_in) ^ A ^ B is the carry into limb k (carry-lookahead with
// ballots).  Groups of 32 limbs compose as maps {0, 1} -> {0, 1} scanned by
// warp shuffles; CTAs likewise (k_settle).  Nothing waits on another CTA.
#pragma once
#include <cstdint>

namespace ffg {

// A carry map c_in -> c_out on one bit: bit 0 = c_out for c_in 0, bit 1 = for c_in 1.
FFG_DEV_INLINE uint32_t map_apply(uint32_t m, uint32_t c) { return (m >> c) & 1u; }
// g after f (f first).
FFG_DEV_INLINE uint32_t map_then(uint32_t f, uint32_t g) {
    return map_apply(g, f & 1u) | (map_apply(g, (f >> 1) & 1u) << 1);
}
FFG_DEV_INLINE uint32_t map_of_group(uint32_t G, uint32_t P) {
    const uint64_t A = G | P, B = G;
    return (uint32_t)((A + B) >> 32) | ((uint32_t)((A + B + 1) >> 32) << 1);
}

// Inclusive scan of one map per lane over a warp.
FFG_DEV_INLINE uint32_t warp_map_scan(uint32_t m) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        uint32_t f = __shfl_up_sync(0xffffffffu, m, d);
        if (lane >= d) m = map_then(f, m);
    }
    return m;
}

// Resolves the CTA's column sums in shared memory: lo[0..NL) (u64), hi[0..NL)
// (small), and hiprev = hi of the limb below the CTA.  On return lo[j] holds
// the final limb j assuming no carry comes into the CTA; the CTA's carry map
// is returned to thread 0.  NL is a multiple of 32; gmask[] and gmap[] are
// shared scratch of NL/32 words each; blockDim.x a multiple of 32.
FFG_DEV_INLINE uint32_t cta_resolve(uint64_t *lo, const uint32_t *hi, uint32_t hiprev, uint32_t NL,
                                    uint32_t *gG, uint32_t *gP, uint32_t *gin) {
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const uint32_t ngroups = NL / 32;
    // v_j = lo_j + hi_(j-1); generate / propagate ballots per group of 32 limbs
    for (uint32_t q = warp; q < ngroups; q += nw) {
        const uint32_t j = q * 32 + lane;
        const uint64_t h = j ? hi[j - 1] : hiprev;
        const uint64_t v = lo[j] + h;
        const bool gj = v < h, pj = v == ~0ull;
        lo[j] = v;
        const uint32_t G = __ballot_sync(0xffffffffu, gj), P = __ballot_sync(0xffffffffu, pj);
        if (lane == 0) {
            gG[q] = G;
            gP[q] = P;
        }
    }
    __syncthreads();
    // carry into every group: one warp scans the group maps
    uint32_t cta_map = 0;
    if (warp == 0) {
        uint32_t carry = 0; // into the next chunk of 32 groups, for c_in = 0
        uint32_t run = 2;   // map of all groups so far (identity: c -> c)
        for (uint32_t base = 0; base < ngroups; base += 32) {
            const uint32_t q = base + lane;
            uint32_t m = q < ngroups ? map_of_group(gG[q], gP[q]) : 2u;
            uint32_t inc = warp_map_scan(m);
            uint32_t exc = __shfl_up_sync(0xffffffffu, inc, 1);
            if (lane == 0) exc = 2u;
            if (q < ngroups) gin[q] = map_apply(exc, carry);
            const uint32_t tot = __shfl_sync(0xffffffffu, inc, 31);
            carry = map_apply(tot, carry);
            run = map_then(run, tot);
        }
        cta_map = run;
    }
    __syncthreads();
    // add each limb's carry
    for (uint32_t q = warp; q < ngroups; q += nw) {
        const uint32_t G = gG[q], P = gP[q], c = gin[q];
        const uint64_t A = G | P, B = G;
        const uint32_t carries = (uint32_t)((A + B + c) ^ A ^ B);
        const uint32_t j = q * 32 + lane;
        lo[j] += (carries >> lane) & 1u;
    }
    __syncthreads();
    return cta_map;
}

// Carries between CTAs, settled by the CTA that finishes last (all of its
// threads): thread t composes the maps of its run of consecutive CTAs, a
// block-wide scan of those composites gives the carry into every run (carry
// 0 into the first CTA), and each thread walks its run again adding the
// carry into the CTAs that receive one: a carry stops at the first limb that
// does not wrap, almost always the first.  A CTA whose map is the identity
// has every limb 2^64 - 1 (Barrett and Newton combinations produce long such
// runs): the carry zeroes it with stores alone.  A carry still running after
// kSettleWalk limbs of any other CTA is finished by the whole block
// afterwards, 256 limbs at a time, so no thread walks thousands of dependent
// loads.
// Maps and limbs written by other CTAs are read through L2.
constexpr uint32_t kSettleWalk = 8;
constexpr uint32_t kSettleLong = 64;

FFG_DEV_INLINE void settle_cta(uint64_t *out, uint64_t nlimbs, uint32_t cta_limbs, const uint32_t *maps,
                               uint32_t ncta) {
    __shared__ uint32_t wpre[32];
    __shared__ uint64_t long_j[kSettleLong], long_end[kSettleLong];
    __shared__ uint32_t nlong;
    __shared__ uint64_t first_s;
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (threadIdx.x == 0) nlong = 0;
    const uint32_t per = (ncta + blockDim.x - 1) / blockDim.x;
    const uint32_t q0 = min(ncta, threadIdx.x * per), q1 = min(ncta, q0 + per);
    uint32_t run = 2u; // identity: c -> c
    for (uint32_t q = q0; q < q1; q++) run = map_then(run, __ldcg(&maps[q]));
    const uint32_t inc = warp_map_scan(run);
    if (lane == 31) wpre[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        const uint32_t v = warp_map_scan(lane < nw ? wpre[lane] : 2u);
        __syncwarp();
        if (lane < nw) wpre[lane] = v;
    }
    __syncthreads();
    uint32_t exc = __shfl_up_sync(0xffffffffu, inc, 1);
    if (lane == 0) exc = 2u;
    const uint32_t before = warp ? map_then(wpre[warp - 1], exc) : exc;
    uint32_t carry = map_apply(before, 0);
    for (uint32_t q = q0; q < q1; q++) {
        const uint32_t mq = __ldcg(&maps[q]);
        if (carry && mq == 2u) {
            // the identity map: every limb of the CTA is 2^64 - 1, so the
            // carry turns them all to 0 and goes on (stores only, no search)
            const uint64_t end = min(nlimbs, (uint64_t)(q + 1) * cta_limbs);
            for (uint64_t j = (uint64_t)q * cta_limbs; j < end; j++) out[j] = 0;
        } else if (carry) {
            const uint64_t end = min(nlimbs, (uint64_t)(q + 1) * cta_limbs);
            uint64_t j = (uint64_t)q * cta_limbs;
            bool running = true;
            for (uint32_t w = 0; w < kSettleWalk && j < end; w++, j++) {
                const uint64_t v = __ldcg(&out[j]) + 1;
                out[j] = v;
                if (v != 0) {
                    running = false;
                    break;
                }
            }
            if (running && j < end) {
                const uint32_t slot = atomicAdd(&nlong, 1u);
                if (slot < kSettleLong) {
                    long_j[slot] = j;
                    long_end[slot] = end;
                } else { // list full: finish here
                    for (; j < end; j++) {
                        const uint64_t v = __ldcg(&out[j]) + 1;
                        out[j] = v;
                        if (v != 0) break;
                    }
                }
            }
        }
        carry = map_apply(mq, carry);
    }
    __syncthreads();
    // the long carries, one at a time by the whole block: limbs before the
    // first one that is not 2^64 - 1 become 0, that one gains 1
    const uint32_t nl = min(nlong, kSettleLong);
    for (uint32_t e = 0; e < nl; e++) {
        const uint64_t end = long_end[e];
        for (uint64_t base = long_j[e]; base < end; base += blockDim.x) {
            if (threadIdx.x == 0) first_s = ~0ull;
            __syncthreads();
            const uint64_t j = base + threadIdx.x;
            const uint64_t v = j < end ? __ldcg(&out[j]) : 0;
            if (j < end && v != ~0ull) atomicMin((unsigned long long *)&first_s, (unsigned long long)j);
            __syncthreads();
            const uint64_t first = first_s;
            if (j < end && j <= first) out[j] = j == first ? v + 1 : 0;
            __syncthreads(); // first_s is reused
            if (first != ~0ull) break;
        }
    }
    __syncthreads();
}

// Called by every CTA of a launch after its limbs and map are written:
// true in the one CTA that takes the last of ncta tickets.
FFG_DEV_INLINE bool last_cta(uint32_t *ticket, uint32_t ncta) {
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(ticket, 1u) == ncta - 1;
    __syncthreads();
    if (last) __threadfence();
    return last;
}

} // namespace ffg
