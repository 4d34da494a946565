// The four-step row pass with its shape fixed at compile time, for rows of
// C = 2^CLG words (9 <= CLG <= 13).
//
// A row is C / 32 threads; a CTA holds up to 256 / (C / 32) rows, fewer when
// that would leave SMs idle (the launch picks the rows per CTA).
// The forward transform of a row is three radix steps of decimation in
// frequency (the last two may merge into one when CLG <= 10):
//   A: radix 2^MA at stride SA = C / 2^MA, straight from global memory;
//   B: radix 2^MB at stride 32, blocks of 32 2^MB words;
//   C: radix 32 at stride 1 (no step twiddles).
// Step C, the pointwise product and the first inverse step (radix 32 at
// stride 1, decimation in time) run on the same 32 registers of a thread
// with no shared-memory round trip in between; then B^-1, and A^-1 ends with
// the four-step twiddle ω_L^-(n2 k1) and the store of the row.  Every shared
// address is a compile-time offset from one base per group, and all strides
// are multiples of 32 (or 1, for step C) on padded lines (pad(i) = i + i/32),
// so no access has a bank conflict.
//
// It computes the same residues as the generic row pass of ffg_ntt.cu
// (k_row_conv, mode ROW_CONV): the order of the frequencies between the
// forward and the inverse differs, but the pointwise product does not care.
#include "ffg_internal.h"
#include "ffg_lines.cuh"

namespace ffg {

template <int CLG> struct RowShape;
template <> struct RowShape<9> { static constexpr int MA = 0, MB = 4; };
template <> struct RowShape<10> { static constexpr int MA = 0, MB = 5; };
template <> struct RowShape<11> { static constexpr int MA = 3, MB = 3; };
template <> struct RowShape<12> { static constexpr int MA = 4, MB = 3; };
template <> struct RowShape<13> { static constexpr int MA = 4, MB = 4; };

constexpr uint32_t cx_line_stride(uint32_t N) {
    return (((N + (N - 1) / 32 + 1) + 31) & ~31u) + 1;
}

template <int CLG> struct RowGeo {
    static constexpr int MA = RowShape<CLG>::MA, MB = RowShape<CLG>::MB;
    static constexpr uint32_t C = 1u << CLG;
    static constexpr uint32_t T = C / 32;          // threads per row
    static constexpr uint32_t ROWS = 256 / T;      // most rows per CTA
    static constexpr uint32_t RA = 1u << MA, RB = 1u << MB;
    static constexpr uint32_t SA = C >> MA;        // stride of step A
    static constexpr uint32_t SAP = SA + SA / 32;  // its padded distance
    static constexpr uint32_t GA = 32 >> MA;       // step-A groups per thread
    static constexpr uint32_t NB = 32 * RB;        // block of step B
    static constexpr uint32_t NBP = NB + NB / 32;
    static constexpr uint32_t GB = 32 >> MB;       // step-B groups per thread
    static constexpr uint32_t LS = cx_line_stride(C); // shared words per line
    static_assert(MA + MB + 5 == CLG, "three steps cover the row");
    static_assert(T * GB * RB == C && (MA == 0 || T * GA * RA == C), "every word in one group per step");
};

// ω_L^-(k1 n2) in Montgomery form for n2 = n0 + d t, t = 0, 1, ...: a running
// product (the inverse four-step twiddle of the generic row pass).
template <int PI>
struct BackTwiddle {
    uint32_t cur, step;
    FFG_DEV_INLINE BackTwiddle(const PrimeDev &P, const FourStep &G, uint32_t k1, uint32_t n0, uint32_t d) {
        const uint64_t e0 = (uint64_t)n0 * k1 % G.L * G.mstep, e1 = (uint64_t)d * k1 % G.L * G.mstep;
        cur = twm<PI>(P, e0 ? FFG_M - e0 : 0);
        step = twm<PI>(P, e1 ? FFG_M - e1 : 0);
    }
    FFG_DEV_INLINE uint32_t apply(uint32_t x) {
        const uint32_t r = mo<PI>(x, cur);
        cur = mo<PI>(cur, step);
        return r;
    }
};

// Forward step A of one operand: global row g -> padded shared line s.
template <int PI, int CLG>
FFG_DEV_INLINE void row_fwd_a(const uint32_t *__restrict__ g, uint32_t *__restrict__ s, uint32_t tau,
                              const uint2 *__restrict__ tw) {
    using Q = RowGeo<CLG>;
#pragma unroll 1
    for (uint32_t k = 0; k < Q::GA; k++) {
        const uint32_t j = tau + Q::T * k;
        uint32_t x[Q::RA];
#pragma unroll
        for (uint32_t t = 0; t < Q::RA; t++) x[t] = g[j + Q::SA * t];
        dft_dif<PI, Q::MA>(x);
#pragma unroll
        for (uint32_t t = 1; t < Q::RA; t++) x[t] = sh<PI>(x[t], __ldg(&tw[(t - 1) * Q::SA + j]));
        uint32_t *d = s + j + (j >> 5);
#pragma unroll
        for (uint32_t t = 0; t < Q::RA; t++) d[t * Q::SAP] = x[t];
    }
}

// Forward step B of one operand: from the padded line s (or, with no step A,
// from the global row g) back into s.
template <int PI, int CLG, bool FROM_G>
FFG_DEV_INLINE void row_fwd_b(const uint32_t *__restrict__ g, uint32_t *__restrict__ s, uint32_t tau,
                              const uint2 *__restrict__ tw) {
    using Q = RowGeo<CLG>;
    // with 32 or more threads a row, a thread's groups share j (and twiddles)
    constexpr bool JFIX = Q::T % 32 == 0;
    uint2 w[Q::RB - 1];
    if (JFIX) {
#pragma unroll
        for (uint32_t t = 1; t < Q::RB; t++) w[t - 1] = __ldg(&tw[(t - 1) * 32 + (tau & 31)]);
    }
#pragma unroll 1
    for (uint32_t k = 0; k < Q::GB; k++) {
        const uint32_t gi = tau + Q::T * k, b = gi >> 5, j = gi & 31;
        if (!JFIX) {
#pragma unroll
            for (uint32_t t = 1; t < Q::RB; t++) w[t - 1] = __ldg(&tw[(t - 1) * 32 + j]);
        }
        uint32_t *d = s + b * Q::NBP + j;
        uint32_t x[Q::RB];
        if (FROM_G) {
            const uint32_t *src = g + b * Q::NB + j;
#pragma unroll
            for (uint32_t t = 0; t < Q::RB; t++) x[t] = src[32 * t];
        } else {
#pragma unroll
            for (uint32_t t = 0; t < Q::RB; t++) x[t] = d[33 * t];
        }
        dft_dif<PI, Q::MB>(x);
#pragma unroll
        for (uint32_t t = 1; t < Q::RB; t++) x[t] = sh<PI>(x[t], w[t - 1]);
#pragma unroll
        for (uint32_t t = 0; t < Q::RB; t++) d[33 * t] = x[t];
    }
}

template <int PI, int CLG, bool SQ>
FFG_DEV_INLINE void row2_body(const PrimeDev &P, const FourStep &G, const FSJob &J, uint32_t *smem) {
    using Q = RowGeo<CLG>;
    const uint32_t r = threadIdx.x / Q::T, tau = threadIdx.x % Q::T;
    const uint32_t pos = blockIdx.x * (blockDim.x / Q::T) + r;
    const size_t rowoff = (size_t)PI * G.L + (size_t)pos * Q::C;
    uint32_t *ya = J.ya + rowoff;
    const uint32_t *yb = SQ ? ya : J.yb + rowoff;
    uint32_t *sa = smem + r * (SQ ? 1 : 2) * Q::LS;
    uint32_t *sb = sa + Q::LS;
    const uint2 *twA = P.stw + c_lines.tw_off[(5 + Q::MB) * 6 + Q::MA];
    const uint2 *twB = P.stw + c_lines.tw_off[5 * 6 + Q::MB];

    if (Q::MA) {
        row_fwd_a<PI, CLG>(ya, sa, tau, twA);
        if (!SQ) row_fwd_a<PI, CLG>(yb, sb, tau, twA);
        __syncthreads();
        row_fwd_b<PI, CLG, false>(ya, sa, tau, twB);
        if (!SQ) row_fwd_b<PI, CLG, false>(yb, sb, tau, twB);
    } else {
        row_fwd_b<PI, CLG, true>(ya, sa, tau, twB);
        if (!SQ) row_fwd_b<PI, CLG, true>(yb, sb, tau, twB);
    }
    __syncthreads();

    // step C, the pointwise product and C^-1 on registers
    {
        uint32_t x[32];
        uint32_t *d = sa + 33 * tau;
        if (!SQ) {
            uint32_t *e = sb + 33 * tau;
#pragma unroll
            for (int t = 0; t < 32; t++) x[t] = e[t];
            dft_dif<PI, 5>(x);
#pragma unroll
            for (int t = 0; t < 32; t++) e[t] = x[t]; // read back below by this thread only
        }
#pragma unroll
        for (int t = 0; t < 32; t++) x[t] = d[t];
        dft_dif<PI, 5>(x);
        if (SQ) {
#pragma unroll
            for (int t = 0; t < 32; t++) x[t] = mo<PI>(x[t], x[t]);
        } else {
            const uint32_t *e = sb + 33 * tau;
#pragma unroll
            for (int t = 0; t < 32; t++) x[t] = mo<PI>(x[t], e[t]);
        }
        dft_dit<PI, 5>(x);
#pragma unroll
        for (int t = 0; t < 32; t++) d[t] = x[t];
    }
    __syncthreads();

    const uint32_t k1 = freq_of(pos, G.rn, G.r3);
    // B^-1 (the last step when there is no step A: then it stores the row)
    {
        const uint2 *itwB = P.istw + c_lines.tw_off[5 * 6 + Q::MB];
        constexpr bool JFIX = Q::T % 32 == 0;
        uint2 w[Q::RB - 1];
        if (JFIX) {
#pragma unroll
            for (uint32_t t = 1; t < Q::RB; t++) w[t - 1] = __ldg(&itwB[(t - 1) * 32 + (tau & 31)]);
        }
#pragma unroll 1
        for (uint32_t k = 0; k < Q::GB; k++) {
            const uint32_t gi = tau + Q::T * k, b = gi >> 5, j = gi & 31;
            if (!JFIX) {
#pragma unroll
                for (uint32_t t = 1; t < Q::RB; t++) w[t - 1] = __ldg(&itwB[(t - 1) * 32 + j]);
            }
            uint32_t *d = sa + b * Q::NBP + j;
            uint32_t x[Q::RB];
#pragma unroll
            for (uint32_t t = 0; t < Q::RB; t++) x[t] = d[33 * t];
#pragma unroll
            for (uint32_t t = 1; t < Q::RB; t++) x[t] = sh<PI>(x[t], w[t - 1]);
            dft_dit<PI, Q::MB>(x);
            if (Q::MA) {
#pragma unroll
                for (uint32_t t = 0; t < Q::RB; t++) d[33 * t] = x[t];
            } else {
                BackTwiddle<PI> bt(P, G, k1, b * Q::NB + j, 32);
                uint32_t *o = ya + b * Q::NB + j;
#pragma unroll
                for (uint32_t t = 0; t < Q::RB; t++) o[32 * t] = bt.apply(x[t]);
            }
        }
    }
    if (!Q::MA) return;
    __syncthreads();

    // A^-1, the four-step twiddle and the store
    const uint2 *itwA = P.istw + c_lines.tw_off[(5 + Q::MB) * 6 + Q::MA];
#pragma unroll 1
    for (uint32_t k = 0; k < Q::GA; k++) {
        const uint32_t j = tau + Q::T * k;
        const uint32_t *d = sa + j + (j >> 5);
        uint32_t x[Q::RA];
#pragma unroll
        for (uint32_t t = 0; t < Q::RA; t++) x[t] = d[t * Q::SAP];
#pragma unroll
        for (uint32_t t = 1; t < Q::RA; t++) x[t] = sh<PI>(x[t], __ldg(&itwA[(t - 1) * Q::SA + j]));
        dft_dit<PI, Q::MA>(x);
        BackTwiddle<PI> bt(P, G, k1, j, Q::SA);
#pragma unroll
        for (uint32_t t = 0; t < Q::RA; t++) ya[j + Q::SA * t] = bt.apply(x[t]);
    }
}

template <int CLG, bool SQ>
__global__ void __launch_bounds__(256, (CLG == 10 && !SQ) ? 2 : 3) k_row2(Primes3 P3, FourStep G, FSJobs jobs) {
    extern __shared__ uint32_t smem[];
    __shared__ FSJob J;
    if (threadIdx.x == 0) J = jobs.ext ? jobs.ext[blockIdx.z] : jobs.j[blockIdx.z < FFG_FS_JOBS ? blockIdx.z : 0];
    __syncthreads();
    switch (blockIdx.y + G.prime0) {
    case 0: row2_body<0, CLG, SQ>(P3.pr[0], G, J, smem); break;
    case 1: row2_body<1, CLG, SQ>(P3.pr[1], G, J, smem); break;
    default: row2_body<2, CLG, SQ>(P3.pr[2], G, J, smem); break;
    }
}

template <int CLG, bool SQ>
static cudaError_t launch_row2_t(const Primes3 &P3, const FourStep &G, const FSJobs &jobs, uint32_t njobs,
                                 cudaStream_t st) {
    using Q = RowGeo<CLG>;
    const size_t smax = (size_t)Q::ROWS * (SQ ? 1 : 2) * Q::LS * sizeof(uint32_t);
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(k_row2<CLG, SQ>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smax);
        if (e) return e;
        attr = true;
    }
    // rows per CTA: as many as fit 256 threads, halved while the launch would
    // have fewer than three CTAs per SM (short rows of a mid-size product)
    uint32_t rows = Q::ROWS;
    while (rows > 1 && (uint64_t)(G.R / rows) * G.nprimes * njobs < 3 * 148) rows >>= 1;
    while (rows > 1 && G.R % rows) rows >>= 1;
    const size_t sm = (size_t)rows * (SQ ? 1 : 2) * Q::LS * sizeof(uint32_t);
    k_row2<CLG, SQ><<<dim3(G.R / rows, G.nprimes, njobs), rows * Q::T, sm, st>>>(P3, G, jobs);
    return cudaGetLastError();
}

// This unit's copy of the line-transform constants (each CUDA unit has its
// own constant bank); set once with the others.
cudaError_t set_line_consts_rows(const LineConsts &h) { return cudaMemcpyToSymbol(c_lines, &h, sizeof h); }

// Whether the fixed-shape row pass takes this geometry (ROW_CONV rows of
// 2^9 .. 2^13 words).
bool row2_ok(const FourStep &G) { return G.mode == ROW_CONV && G.c >= 9 && G.c <= 13; }

cudaError_t launch_row2(const Primes3 &P3, const FourStep &G, const FSJobs &jobs, uint32_t njobs, cudaStream_t st) {
    const bool sq = G.square != 0;
    switch (G.c) {
    case 9: return sq ? launch_row2_t<9, true>(P3, G, jobs, njobs, st) : launch_row2_t<9, false>(P3, G, jobs, njobs, st);
    case 10: return sq ? launch_row2_t<10, true>(P3, G, jobs, njobs, st) : launch_row2_t<10, false>(P3, G, jobs, njobs, st);
    case 11: return sq ? launch_row2_t<11, true>(P3, G, jobs, njobs, st) : launch_row2_t<11, false>(P3, G, jobs, njobs, st);
    case 12: return sq ? launch_row2_t<12, true>(P3, G, jobs, njobs, st) : launch_row2_t<12, false>(P3, G, jobs, njobs, st);
    default: return sq ? launch_row2_t<13, true>(P3, G, jobs, njobs, st) : launch_row2_t<13, false>(P3, G, jobs, njobs, st);
    }
}

} // namespace ffg
