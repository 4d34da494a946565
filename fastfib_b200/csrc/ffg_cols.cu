// The four-step column passes with the column length fixed at compile time,
// for columns of R = 2^RN or 3 2^RN words (6 <= RN <= 13).
//
// A CTA holds a tile of wc columns x R rows in shared memory, one padded
// line per column.  The length-2^RN transform of each column (of each of its
// three blocks of 2^RN words when R = 3 2^RN) is three radix steps
// (decimation in frequency forward, in time inverse):
//   A: radix 2^MA at stride 2^RN / 2^MA (absent when RN <= 9),
//   B: radix 2^MB at stride 32,
//   C: radix 32 at stride 1 (no step twiddles);
// with R = 3 2^RN a radix-3 step at stride 2^RN comes first (forward) or
// last (inverse), as in the generic line transforms (r3_dif / r3_dit).
// k_col_fwd2: the first step reads the operand's digits straight from its
//   limbs (the reference's Src reader, src/ntt_kernels.c:29-74, one digit per
//   word), step C ends with the four-step twiddle ω_L^(n2 k1) and stores the
//   residues row-major, as the generic column pass (ffg_ntt.cu k_col_fwd).
// k_col_inv2: step C^-1 reads the row pass's output straight from global
//   memory, the last step scales by 2^32 / L and stores (or adds into the
//   split's residues), as k_col_inv.
// Each step maps thread slots p = threadIdx.x + blockDim.x k to (column p mod wc,
// group p / wc), so a warp's global accesses cover min(wc, 32) consecutive
// words of each row it touches, and consecutive lines start 32 / min(wc, 32)
// banks apart, so no shared access has a bank conflict.
#include "ffg_internal.h"
#include "ffg_lines.cuh"

namespace ffg {

__host__ __device__ constexpr int brev5(int u) { return ((u & 1) << 4) | ((u & 2) << 2) | (u & 4) | ((u & 8) >> 2) | ((u & 16) >> 4); }

template <int RN> struct ColShape;
template <> struct ColShape<6> { static constexpr int MA = 0, MB = 1; };
template <> struct ColShape<7> { static constexpr int MA = 0, MB = 2; };
template <> struct ColShape<8> { static constexpr int MA = 0, MB = 3; };
template <> struct ColShape<9> { static constexpr int MA = 0, MB = 4; };
template <> struct ColShape<10> { static constexpr int MA = 2, MB = 3; };
template <> struct ColShape<11> { static constexpr int MA = 3, MB = 3; };
template <> struct ColShape<12> { static constexpr int MA = 4, MB = 3; };
template <> struct ColShape<13> { static constexpr int MA = 4, MB = 4; };

template <int RN> struct ColGeo {
    static constexpr int MA = ColShape<RN>::MA, MB = ColShape<RN>::MB;
    static constexpr uint32_t R = 1u << RN;
    static constexpr uint32_t RA = 1u << MA, RB = 1u << MB;
    static constexpr uint32_t SA = R >> MA, SAP = SA + SA / 32;
    static constexpr uint32_t NB = 32 * RB, NBP = NB + NB / 32;
    static_assert(MA + MB + 5 == RN, "three steps cover the column");
};

// Shared words per column line: the padded length, rounded so that
// consecutive lines start 32 / min(wc, 32) banks apart.
__host__ __device__ inline uint32_t col2_stride(uint32_t R, uint32_t wc) {
    const uint32_t wl = wc < 32 ? wc : 32;
    return ((R + R / 32 + 31) & ~31u) + 32 / wl;
}

// What the first step of a forward column tile reads: the operand's digits.
struct ColSrc {
    const uint64_t *src;
    uint64_t ns, cs, off;
    uint32_t w, C, c0, wc, wlg, LS;
};

// The raw limb words behind one digit: the 32-bit word itself for 32-bit
// digits, else the two 64-bit limbs the digit may straddle.
template <bool W32> struct DigitRaw;
template <> struct DigitRaw<true> {
    uint32_t v;
    FFG_DEV_INLINE void fetch(const ColSrc &S, uint64_t i, bool ok) {
        // digit i is 32-bit word off + i of the limbs
        const uint64_t q = S.off + i;
        v = ok && i < S.cs && (q >> 1) < S.ns ? __ldg((const uint32_t *)S.src + q) : 0u;
    }
    template <int PI> FFG_DEV_INLINE uint32_t residue(const ColSrc &, uint64_t, const PrimeDev &) const {
        constexpr uint32_t p = kPrimeC[PI];
        uint32_t l = v;
        l = min(l, l - p);
        return min(l, l - p);
    }
};
template <> struct DigitRaw<false> {
    uint64_t lo, hi;
    FFG_DEV_INLINE void fetch(const ColSrc &S, uint64_t i, bool ok) {
        const uint64_t bit = (S.off + i) * S.w, q = bit >> 6;
        const uint32_t sft = (uint32_t)(bit & 63);
        ok = ok && i < S.cs;
        lo = ok && q < S.ns ? __ldg(&S.src[q]) : 0;
        hi = ok && sft + S.w > 64 && q + 1 < S.ns ? __ldg(&S.src[q + 1]) : 0;
    }
    template <int PI> FFG_DEV_INLINE uint32_t residue(const ColSrc &S, uint64_t i, const PrimeDev &P) const {
        constexpr uint32_t p = kPrimeC[PI];
        const uint32_t sft = (uint32_t)(((S.off + i) * S.w) & 63);
        const uint64_t v = (sft ? (lo >> sft) | (hi << (64 - sft)) : lo) & ((1ull << S.w) - 1);
        uint32_t l = (uint32_t)v;
        l = min(l, l - p);
        l = min(l, l - p);
        return ad<PI>(l, sh<PI>((uint32_t)(v >> 32), make_uint2(P.c32, P.c32s)));
    }
};

// The first step of a power-of-two forward column tile, straight from the
// digits, when only rows below NZ * (its stride) can be nonzero (a product's
// operands fill at most the lower half of the transform, a short operand much
// less): the zero slots are neither read nor transformed (dft_dif_nz).
// Step A (radix 2^MA at stride 2^RN / 2^MA) when MA > 0, else step B (radix
// 2^MB at stride 32, one block).  The limb words of a thread's next slot are
// loaded before its current slot is transformed, so each thread keeps two
// slots' loads in flight: the strided column reads are latency-bound.
template <int PI, int RN, int NZ, bool W32>
FFG_DEV_INLINE void col_fwd2_first_w(const PrimeDev &P, const ColSrc &S, uint32_t *smem) {
    using Q = ColGeo<RN>;
    constexpr bool A = Q::MA > 0;
    constexpr int M = A ? Q::MA : Q::MB;
    constexpr uint32_t RM = 1u << M, STRIDE = A ? Q::SA : 32, DP = A ? Q::SAP : 33;
    const uint32_t wc = S.wc, wlg = S.wlg;
    const uint32_t slots = wc * STRIDE;
    const uint2 *tw = P.stw + c_lines.tw_off[(A ? RN - Q::MA : 5) * 6 + M];
    auto index = [&](uint32_t sl, uint32_t t) -> uint64_t {
        return (uint64_t)((sl >> wlg) + STRIDE * t) * S.C + S.c0 + (sl & (wc - 1));
    };
    // prefetch while the two slots' words fit the registers (16 words for
    // 32-bit digits, 4 digits' limb pairs otherwise)
    constexpr bool PF = W32 ? NZ <= 16 : NZ <= 4;
    DigitRaw<W32> cur[NZ];
    if (PF) {
#pragma unroll
        for (uint32_t t = 0; t < (uint32_t)NZ; t++) cur[t].fetch(S, index(threadIdx.x, t), threadIdx.x < slots);
    }
#pragma unroll 1
    for (uint32_t sl = threadIdx.x; sl < slots; sl += blockDim.x) {
        DigitRaw<W32> nxt[PF ? NZ : 1];
        const uint32_t sn = sl + blockDim.x;
        if (PF) {
#pragma unroll
            for (uint32_t t = 0; t < (uint32_t)NZ; t++) nxt[t < (PF ? NZ : 1) ? t : 0].fetch(S, index(sn, t), sn < slots);
        } else {
#pragma unroll
            for (uint32_t t = 0; t < (uint32_t)NZ; t++) cur[t].fetch(S, index(sl, t), true);
        }
        const uint32_t c = sl & (wc - 1), j = sl >> wlg;
        uint32_t x[RM];
#pragma unroll
        for (uint32_t t = 0; t < RM; t++) x[t] = t < (uint32_t)NZ ? cur[t < (uint32_t)NZ ? t : 0].template residue<PI>(S, index(sl, t), P) : 0u;
        dft_dif_nz<PI, M, NZ>(x);
#pragma unroll
        for (uint32_t t = 1; t < RM; t++) x[t] = sh<PI>(x[t], __ldg(&tw[(t - 1) * STRIDE + j]));
        uint32_t *d = smem + c * S.LS + j + (A ? (j >> 5) : 0);
#pragma unroll
        for (uint32_t t = 0; t < RM; t++) d[t * DP] = x[t];
        if (PF) {
#pragma unroll
            for (uint32_t t = 0; t < (uint32_t)NZ; t++) cur[t] = nxt[t < (PF ? NZ : 1) ? t : 0];
        }
    }
}

template <int PI, int RN, int NZ>
FFG_DEV_INLINE void col_fwd2_first(const PrimeDev &P, const ColSrc &S, uint32_t *smem) {
    if (S.w == 32) col_fwd2_first_w<PI, RN, NZ, true>(P, S, smem);
    else col_fwd2_first_w<PI, RN, NZ, false>(P, S, smem);
}

// The radix-3 first step (stride 2^RN) of a forward column tile of 3 2^RN
// rows, straight from the digits, when only the first NB of its three blocks
// can hold nonzero rows (NB = 1: y0 = x0, y1 = x0 w^j, y2 = x0 w^2j; NB = 2:
// x2 = 0), with the next slot's limb words loaded before the current slot is
// transformed, as col_fwd2_first_w.
template <int PI, int RN, int NB, bool W32>
FFG_DEV_INLINE void col_fwd2_first_r3(const PrimeDev &P, const ColSrc &S, uint32_t *smem) {
    using Q = ColGeo<RN>;
    constexpr uint32_t p = kPrimeC[PI], BP = Q::R + Q::R / 32;
    constexpr bool PF = W32 || NB <= 2;
    const uint32_t wc = S.wc, wlg = S.wlg;
    const uint32_t slots = wc * Q::R;
    auto index = [&](uint32_t sl, uint32_t q) -> uint64_t {
        return (uint64_t)((sl >> wlg) + Q::R * q) * S.C + S.c0 + (sl & (wc - 1));
    };
    DigitRaw<W32> cur[NB];
    if (PF) {
#pragma unroll
        for (int q = 0; q < NB; q++) cur[q].fetch(S, index(threadIdx.x, q), threadIdx.x < slots);
    }
#pragma unroll 1
    for (uint32_t sl = threadIdx.x; sl < slots; sl += blockDim.x) {
        DigitRaw<W32> nxt[PF ? NB : 1];
        const uint32_t sn = sl + blockDim.x;
        if (PF) {
#pragma unroll
            for (int q = 0; q < NB; q++) nxt[PF ? q : 0].fetch(S, index(sn, q), sn < slots);
        } else {
#pragma unroll
            for (int q = 0; q < NB; q++) cur[q].fetch(S, index(sl, q), true);
        }
        const uint32_t c = sl & (wc - 1), j = sl >> wlg;
        const uint32_t x0 = cur[0].template residue<PI>(S, index(sl, 0), P);
        const uint32_t x1 = NB > 1 ? cur[NB > 1 ? 1 : 0].template residue<PI>(S, index(sl, 1), P) : 0u;
        const uint32_t x2 = NB > 2 ? cur[NB > 2 ? 2 : 0].template residue<PI>(S, index(sl, 2), P) : 0u;
        const uint4 t = __ldg(&P.r3f[Q::R + j]);
        uint32_t *d = smem + c * S.LS + j + (j >> 5);
        if (NB == 1) {
            d[0] = x0;
            d[BP] = sh<PI>(x0, make_uint2(t.x, t.y));
            d[2 * BP] = sh<PI>(x0, make_uint2(t.z, t.w));
        } else {
            const uint32_t u = sh<PI>(x1 - x2 + p, c_lines.w3[PI]);
            d[0] = ad<PI>(ad<PI>(x0, x1), x2);
            d[BP] = sh<PI>(ad<PI>(sb<PI>(x0, x2), u), make_uint2(t.x, t.y));
            d[2 * BP] = sh<PI>(sb<PI>(sb<PI>(x0, x1), u), make_uint2(t.z, t.w));
        }
        if (PF) {
#pragma unroll
            for (int q = 0; q < NB; q++) cur[q] = nxt[PF ? q : 0];
        }
    }
}

// col_fwd2_first for the least power of two NZ covering nzt slots.
template <int PI, int RN>
FFG_DEV_INLINE void col_fwd2_first_any(const PrimeDev &P, const ColSrc &S, uint32_t *smem, uint32_t nzt) {
    using Q = ColGeo<RN>;
    constexpr int M = Q::MA ? Q::MA : Q::MB;
    if (nzt <= 1) col_fwd2_first<PI, RN, 1>(P, S, smem);
    else if (nzt <= 2 || M < 2) col_fwd2_first<PI, RN, (M >= 1 ? 2 : 1)>(P, S, smem);
    else if (nzt <= 4 || M < 3) col_fwd2_first<PI, RN, (M >= 2 ? 4 : 1)>(P, S, smem);
    else if (nzt <= 8 || M < 4) col_fwd2_first<PI, RN, (M >= 3 ? 8 : 1)>(P, S, smem);
    else if (nzt <= 16 || M < 5) col_fwd2_first<PI, RN, (M >= 4 ? 16 : 1)>(P, S, smem);
    else col_fwd2_first<PI, RN, (M >= 5 ? 32 : 1)>(P, S, smem);
}

template <int PI, int RN, bool R3>
FFG_DEV_INLINE void col_fwd2_body(const PrimeDev &P, const FourStep &G, const FSJob &J, uint32_t *smem) {
    using Q = ColGeo<RN>;
    constexpr uint32_t NBLK = R3 ? 3 : 1, BP = Q::R + Q::R / 32; // blocks and padded block length
    const uint32_t op = G.square ? 0 : (blockIdx.z & 1);
    const uint32_t C = 1u << G.c, wc = G.wc, wlg = G.wc_lg, LS = col2_stride(NBLK * Q::R, wc);
    const uint32_t c0 = blockIdx.x * wc;
    const uint64_t *src = op ? J.b : J.a;
    const uint64_t ns = op ? J.nb : J.na, cs = op ? J.cb : J.ca, off = op ? J.off_b : J.off_a;
    const uint32_t w = J.width;

    // rows at or past rows_nz are zero in every column of the tile
    const uint64_t avail = (ns * 64 + w - 1) / w; // digits that start inside the limbs
    const uint64_t lim = cs < (avail > off ? avail - off : 0) ? cs : (avail > off ? avail - off : 0);
    const uint64_t rows_nz = lim > c0 ? (lim - c0 + C - 1) / C : 0;
    if (R3) { // radix 3 at stride 2^RN, straight from the digits
        const ColSrc S{src, ns, cs, off, w, C, c0, wc, wlg, LS};
        const uint32_t nb = rows_nz <= Q::R ? 1 : rows_nz <= 2 * Q::R ? 2 : 3;
        if (w == 32) {
            if (nb == 1) col_fwd2_first_r3<PI, RN, 1, true>(P, S, smem);
            else if (nb == 2) col_fwd2_first_r3<PI, RN, 2, true>(P, S, smem);
            else col_fwd2_first_r3<PI, RN, 3, true>(P, S, smem);
        } else {
            if (nb == 1) col_fwd2_first_r3<PI, RN, 1, false>(P, S, smem);
            else if (nb == 2) col_fwd2_first_r3<PI, RN, 2, false>(P, S, smem);
            else col_fwd2_first_r3<PI, RN, 3, false>(P, S, smem);
        }
        __syncthreads();
    }
    if (!R3) {
        const uint32_t stride = Q::MA ? Q::SA : 32;
        const uint32_t nzt = (uint32_t)((rows_nz + stride - 1) / stride);
        const ColSrc S{src, ns, cs, off, w, C, c0, wc, wlg, LS};
        col_fwd2_first_any<PI, RN>(P, S, smem, nzt);
        __syncthreads();
    }
    if (Q::MA && R3) {
        const uint2 *tw = P.stw + c_lines.tw_off[(RN - Q::MA) * 6 + Q::MA];
        const uint32_t slots = wc * NBLK * Q::SA;
#pragma unroll 1
        for (uint32_t s = threadIdx.x; s < slots; s += blockDim.x) {
            const uint32_t c = s & (wc - 1), g = s >> wlg, q = g >> (RN - Q::MA), j = g & (Q::SA - 1);
            uint32_t *d = smem + c * LS + q * BP + j + (j >> 5);
            uint32_t x[Q::RA];
#pragma unroll
            for (uint32_t t = 0; t < Q::RA; t++) x[t] = d[t * Q::SAP];
            dft_dif<PI, Q::MA>(x);
#pragma unroll
            for (uint32_t t = 1; t < Q::RA; t++) x[t] = sh<PI>(x[t], __ldg(&tw[(t - 1) * Q::SA + j]));
#pragma unroll
            for (uint32_t t = 0; t < Q::RA; t++) d[t * Q::SAP] = x[t];
        }
        __syncthreads();
    }
    if (Q::MA || R3) {
        const uint2 *tw = P.stw + c_lines.tw_off[5 * 6 + Q::MB];
        const uint32_t slots = wc * NBLK * (Q::R / Q::RB);
#pragma unroll 1
        for (uint32_t s = threadIdx.x; s < slots; s += blockDim.x) {
            // blocks of NB words run on through the radix-3 blocks (NB divides 2^RN)
            const uint32_t c = s & (wc - 1), g = s >> wlg, b = g >> 5, j = g & 31;
            uint32_t *d = smem + c * LS + b * Q::NBP + j;
            uint32_t x[Q::RB];
#pragma unroll
            for (uint32_t t = 0; t < Q::RB; t++) x[t] = d[33 * t];
            dft_dif<PI, Q::MB>(x);
#pragma unroll
            for (uint32_t t = 1; t < Q::RB; t++) x[t] = sh<PI>(x[t], __ldg(&tw[(t - 1) * 32 + j]));
#pragma unroll
            for (uint32_t t = 0; t < Q::RB; t++) d[33 * t] = x[t];
        }
    }
    __syncthreads();
    // step C, then ω_L^(n2 k1): position q 2^RN + 32 b + t holds frequency
    // k1 = q + m brev_RN(32 b + t) = q + m (brev_5(t) 2^(RN - 5) + brev_(RN - 5)(b)),
    // m = 3 with the radix-3 step (q its block), else m = 1 and q = 0
    constexpr uint32_t m3 = R3 ? 3 : 1;
    uint32_t *y = (op ? J.yb : J.ya) + (size_t)PI * G.L;
    const uint32_t slots = wc * NBLK * (Q::R / 32);
#pragma unroll 1
    for (uint32_t s = threadIdx.x; s < slots; s += blockDim.x) {
        const uint32_t c = s & (wc - 1), b = s >> wlg, n2 = c0 + c;
        const uint32_t q = b >> (RN - 5), bl = b & ((Q::R >> 5) - 1);
        const uint32_t *d = smem + c * LS + q * BP + 33 * bl;
        uint32_t x[32];
#pragma unroll
        for (int t = 0; t < 32; t++) x[t] = d[t];
        dft_dif<PI, 5>(x);
        const uint32_t bb = __brev(bl) >> (32 - (RN - 5));
        uint32_t cur = twm<PI>(P, (uint64_t)n2 * (q + m3 * bb) % G.L * G.mstep);
        const uint32_t step = twm<PI>(P, ((uint64_t)n2 * m3 << (RN - 5)) % G.L * G.mstep);
        uint32_t *o = y + (size_t)(32 * b) * C + n2;
#pragma unroll
        for (int u = 0; u < 32; u++) {
            const int t = brev5(u); // compile-time after unrolling
            o[(size_t)t * C] = mo<PI>(x[t], cur);
            cur = mo<PI>(cur, step);
        }
    }
}

template <int RN, bool R3>
__global__ void __launch_bounds__(kLineThreads, 3) k_col_fwd2(Primes3 P3, FourStep G, FSJobs jobs) {
    extern __shared__ uint32_t smem[];
    __shared__ FSJob J;
    if (threadIdx.x == 0) {
        const uint32_t i = G.square ? blockIdx.z : (blockIdx.z >> 1);
        J = jobs.ext ? jobs.ext[i] : jobs.j[i < FFG_FS_JOBS ? i : 0];
    }
    __syncthreads();
    switch (blockIdx.y + G.prime0) {
    case 0: col_fwd2_body<0, RN, R3>(P3.pr[0], G, J, smem); break;
    case 1: col_fwd2_body<1, RN, R3>(P3.pr[1], G, J, smem); break;
    default: col_fwd2_body<2, RN, R3>(P3.pr[2], G, J, smem); break;
    }
}

// The final store of the inverse: scaled, written or added into the split's
// residues.
template <int PI>
FFG_DEV_INLINE void col_out(const FourStep &G, const FSJob &J, uint32_t n1, uint32_t n2, uint32_t x, uint2 sc) {
    const size_t at = (size_t)n1 * (1u << G.c) + n2;
    const uint32_t v = sh<PI>(x, sc);
    if (J.yacc) {
        uint32_t *acc = J.yacc + (size_t)PI * J.acc_stride + J.acc_off + at;
        *acc = ad<PI>(*acc, v);
    } else {
        J.ya[(size_t)PI * G.L + at] = v;
    }
}

template <int PI, int RN, bool R3>
FFG_DEV_INLINE void col_inv2_body(const PrimeDev &P, const FourStep &G, const FSJob &J, uint32_t *smem) {
    using Q = ColGeo<RN>;
    constexpr uint32_t NBLK = R3 ? 3 : 1, BP = Q::R + Q::R / 32;
    const uint32_t C = 1u << G.c, wc = G.wc, wlg = G.wc_lg, LS = col2_stride(NBLK * Q::R, wc);
    const uint32_t c0 = blockIdx.x * wc;
    const uint32_t *y = J.ya + (size_t)PI * G.L;
    const uint2 sc = make_uint2(G.scl[PI], G.scls[PI]);
    {
        const uint32_t slots = wc * NBLK * (Q::R / 32);
#pragma unroll 1
        for (uint32_t s = threadIdx.x; s < slots; s += blockDim.x) {
            const uint32_t c = s & (wc - 1), b = s >> wlg;
            const uint32_t q = b >> (RN - 5), bl = b & ((Q::R >> 5) - 1);
            const uint32_t *g = y + (size_t)(32 * b) * C + c0 + c;
            uint32_t x[32];
#pragma unroll
            for (int t = 0; t < 32; t++) x[t] = g[(size_t)t * C];
            dft_dit<PI, 5>(x);
            uint32_t *d = smem + c * LS + q * BP + 33 * bl;
#pragma unroll
            for (int t = 0; t < 32; t++) d[t] = x[t];
        }
    }
    __syncthreads();
    {
        const uint2 *tw = P.istw + c_lines.tw_off[5 * 6 + Q::MB];
        const uint32_t slots = wc * NBLK * (Q::R / Q::RB);
#pragma unroll 1
        for (uint32_t s = threadIdx.x; s < slots; s += blockDim.x) {
            const uint32_t c = s & (wc - 1), g = s >> wlg, b = g >> 5, j = g & 31;
            uint32_t *d = smem + c * LS + b * Q::NBP + j;
            uint32_t x[Q::RB];
#pragma unroll
            for (uint32_t t = 0; t < Q::RB; t++) x[t] = d[33 * t];
#pragma unroll
            for (uint32_t t = 1; t < Q::RB; t++) x[t] = sh<PI>(x[t], __ldg(&tw[(t - 1) * 32 + j]));
            dft_dit<PI, Q::MB>(x);
            if (Q::MA || R3) {
#pragma unroll
                for (uint32_t t = 0; t < Q::RB; t++) d[33 * t] = x[t];
            } else {
#pragma unroll
                for (uint32_t t = 0; t < Q::RB; t++) col_out<PI>(G, J, b * Q::NB + j + 32 * t, c0 + c, x[t], sc);
            }
        }
    }
    if (!Q::MA && !R3) return;
    __syncthreads();
    if (Q::MA) {
        const uint2 *tw = P.istw + c_lines.tw_off[(RN - Q::MA) * 6 + Q::MA];
        const uint32_t slots = wc * NBLK * Q::SA;
#pragma unroll 1
        for (uint32_t s = threadIdx.x; s < slots; s += blockDim.x) {
            const uint32_t c = s & (wc - 1), g = s >> wlg, q = g >> (RN - Q::MA), j = g & (Q::SA - 1);
            uint32_t *d = smem + c * LS + q * BP + j + (j >> 5);
            uint32_t x[Q::RA];
#pragma unroll
            for (uint32_t t = 0; t < Q::RA; t++) x[t] = d[t * Q::SAP];
#pragma unroll
            for (uint32_t t = 1; t < Q::RA; t++) x[t] = sh<PI>(x[t], __ldg(&tw[(t - 1) * Q::SA + j]));
            dft_dit<PI, Q::MA>(x);
            if (R3) {
#pragma unroll
                for (uint32_t t = 0; t < Q::RA; t++) d[t * Q::SAP] = x[t];
            } else {
#pragma unroll
                for (uint32_t t = 0; t < Q::RA; t++) col_out<PI>(G, J, j + Q::SA * t, c0 + c, x[t], sc);
            }
        }
        if (!R3) return;
        __syncthreads();
    }
    // radix 3 at stride 2^RN (the generic r3_dit), scaled and stored
    constexpr uint32_t p = kPrimeC[PI];
    const uint32_t slots = wc * Q::R;
#pragma unroll 1
    for (uint32_t s = threadIdx.x; s < slots; s += blockDim.x) {
        const uint32_t c = s & (wc - 1), j = s >> wlg;
        const uint32_t *d = smem + c * LS + j + (j >> 5);
        const uint4 t = __ldg(&P.r3i[Q::R + j]);
        const uint32_t y0 = d[0];
        const uint32_t z1 = sh<PI>(d[BP], make_uint2(t.x, t.y));
        const uint32_t z2 = sh<PI>(d[2 * BP], make_uint2(t.z, t.w));
        const uint32_t u = sh<PI>(z1 - z2 + p, c_lines.v3[PI]);
        col_out<PI>(G, J, j, c0 + c, ad<PI>(ad<PI>(y0, z1), z2), sc);
        col_out<PI>(G, J, j + Q::R, c0 + c, ad<PI>(sb<PI>(y0, z2), u), sc);
        col_out<PI>(G, J, j + 2 * Q::R, c0 + c, sb<PI>(sb<PI>(y0, z1), u), sc);
    }
}

template <int RN, bool R3>
__global__ void __launch_bounds__(kLineThreads, R3 ? 2 : 3) k_col_inv2(Primes3 P3, FourStep G, FSJobs jobs) {
    extern __shared__ uint32_t smem[];
    __shared__ FSJob J;
    if (threadIdx.x == 0) J = jobs.ext ? jobs.ext[blockIdx.z] : jobs.j[blockIdx.z < FFG_FS_JOBS ? blockIdx.z : 0];
    __syncthreads();
    switch (blockIdx.y + G.prime0) {
    case 0: col_inv2_body<0, RN, R3>(P3.pr[0], G, J, smem); break;
    case 1: col_inv2_body<1, RN, R3>(P3.pr[1], G, J, smem); break;
    default: col_inv2_body<2, RN, R3>(P3.pr[2], G, J, smem); break;
    }
}

cudaError_t set_line_consts_cols(const LineConsts &h) { return cudaMemcpyToSymbol(c_lines, &h, sizeof h); }

static size_t col2_smem(const FourStep &G) { return (size_t)G.wc * col2_stride(G.R, G.wc) * sizeof(uint32_t); }

// Whether the fixed-shape column passes take this geometry: columns of
// 2^6 .. 2^13 words (3 2^6 .. 3 2^12 with the radix-3 step, as far as its
// twiddle tables go), tiles of 8..64
// columns that fit in 110 KB of shared memory.
bool col2_ok(const FourStep &G) {
    return G.rn >= 6 && G.rn <= (G.r3 ? 12u : 13u) && G.wc >= 8 && G.wc <= 64 && G.wc == (1u << G.wc_lg) && G.wc <= (1u << G.c) &&
           col2_smem(G) <= 110 * 1024;
}

template <int RN, bool R3>
static cudaError_t launch_col2_t(bool fwd, const Primes3 &P3, const FourStep &G, const FSJobs &jobs, uint32_t nz,
                                 cudaStream_t st) {
    const void *k = fwd ? (const void *)k_col_fwd2<RN, R3> : (const void *)k_col_inv2<RN, R3>;
    static bool attr[2] = {false, false};
    if (!attr[fwd]) {
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, 110 * 1024);
        if (e) return e;
        attr[fwd] = true;
    }
    const dim3 grid((1u << G.c) / G.wc, G.nprimes, nz);
    // threads per CTA: about one per four groups of the radix-32 step (short
    // columns give a tile few groups; idle threads would only wait)
    const uint32_t groups = G.wc * (uint32_t)(G.R / 32);
    uint32_t threads = groups * 4 < kLineThreads ? groups * 4 : kLineThreads;
    threads = threads < 64 ? 64 : (threads + 31) & ~31u;
    if (fwd) k_col_fwd2<RN, R3><<<grid, threads, col2_smem(G), st>>>(P3, G, jobs);
    else k_col_inv2<RN, R3><<<grid, threads, col2_smem(G), st>>>(P3, G, jobs);
    return cudaGetLastError();
}

template <bool R3>
static cudaError_t launch_col2_r(bool fwd, const Primes3 &P3, const FourStep &G, const FSJobs &jobs, uint32_t nz,
                                 cudaStream_t st) {
    switch (G.rn) {
    case 6: return launch_col2_t<6, R3>(fwd, P3, G, jobs, nz, st);
    case 7: return launch_col2_t<7, R3>(fwd, P3, G, jobs, nz, st);
    case 8: return launch_col2_t<8, R3>(fwd, P3, G, jobs, nz, st);
    case 9: return launch_col2_t<9, R3>(fwd, P3, G, jobs, nz, st);
    case 10: return launch_col2_t<10, R3>(fwd, P3, G, jobs, nz, st);
    case 11: return launch_col2_t<11, R3>(fwd, P3, G, jobs, nz, st);
    case 12: return launch_col2_t<12, R3>(fwd, P3, G, jobs, nz, st);
    default: return launch_col2_t<13, R3>(fwd, P3, G, jobs, nz, st);
    }
}

// nz: grid depth (jobs x operands for the forward pass, jobs for the inverse).
cudaError_t launch_col2(bool fwd, const Primes3 &P3, const FourStep &G, const FSJobs &jobs, uint32_t nz,
                        cudaStream_t st) {
    return G.r3 ? launch_col2_r<true>(fwd, P3, G, jobs, nz, st) : launch_col2_r<false>(fwd, P3, G, jobs, nz, st);
}

} // namespace ffg
