// Line transforms in shared memory, specialised per prime.
//
// A CTA holds `lines` lines (a power of two) of length 3^r3 2^n; line k,
// block q (q < 3 when r3) element i sits at word k * stride + pad((q << n) + i)
// with pad(i) = i + i/32, stride = 1 mod 32.  A forward transform is an
// optional radix-3 DIF step (stride 2^n), then radix-2^M DIF steps on every
// 2^n block following schedule(); the inverse runs the mirror steps in the
// opposite order.
//
// One radix-2^M step at stride S = 2^sl over a block of N = 2^M S words
// takes, for every j < S, the 2^M words j + t S into registers, runs a
// 2^M-point DFT on them (natural order in, bit-reversed out) whose roots are
// the fixed ω_32^e of the prime, and multiplies slot s by the step twiddle
// ω_N^(j brev_M(s)) (one table load per slot, shared by all lines of the CTA
// the thread handles).  Composed, the steps give the DFT in bit-reversed
// order, the same layout as radix-2 decimation in frequency.  The inverse
// step multiplies by ω_N^-(j brev_M(s)) first, then runs the inverse
// in-register DFT (bit-reversed in, natural out).
//
// Every function is a template over the prime index PI, so p and the
// in-register roots are compile-time: p folds into immediates and the roots
// are read as constant-bank operands.  Residues stay canonical in [0, p):
// with p close to 2^31 a lazy [0, 2p) form would overflow 32 bits in x - y + 2p.
#pragma once
#include "ffg_device.cuh"

namespace ffg {

constexpr uint32_t kPrimeC[3] = {2113929217u, 2013265921u, 1811939329u};
constexpr uint32_t kLineThreads = 256; // every line kernel runs 256 threads
constexpr uint32_t kLineThreadsLg = 8;
constexpr int kLineMinBlocks = 3;     // 80 registers a thread

// Filled once per process (set_line_consts in ffg_ntt.cu).
static __constant__ LineConsts c_lines;

template <int PI>
FFG_DEV_INLINE uint32_t ad(uint32_t a, uint32_t b) {
    constexpr uint32_t p = kPrimeC[PI];
    const uint32_t s = a + b;
    return min(s, s - p);
}
template <int PI>
FFG_DEV_INLINE uint32_t sb(uint32_t a, uint32_t b) {
    constexpr uint32_t p = kPrimeC[PI];
    const uint32_t d = a - b;
    return min(d, d + p);
}
// a w mod p for any 32-bit a, (w, floor(w 2^32 / p)) a Shoup pair.
template <int PI>
FFG_DEV_INLINE uint32_t sh(uint32_t a, uint2 w) {
    constexpr uint32_t p = kPrimeC[PI];
    const uint32_t q = __umulhi(a, w.y);
    const uint32_t r = a * w.x - q * p;
    return min(r, r - p);
}
// a b 2^-32 mod p (Montgomery), a, b in [0, p).
template <int PI>
FFG_DEV_INLINE uint32_t mo(uint32_t a, uint32_t b) {
    constexpr uint32_t p = kPrimeC[PI];
    const uint64_t t = (uint64_t)a * b;
    const uint32_t m = (uint32_t)t * c_lines.pinv[PI];
    const uint32_t r = (uint32_t)(t >> 32) - __umulhi(m, p);
    return min(r, r + p);
}

// 2^M-point DFT on registers, decimation in frequency: natural order in,
// slot s holds frequency brev_M(s).  Level l pairs t, t + h (h = 2^(M-1-l))
// with root ω_2h^(t mod h) = ω_32^((t mod h) 16 / h).
template <int PI, int M>
FFG_DEV_INLINE void dft_dif(uint32_t (&x)[1 << M]) {
    constexpr uint32_t p = kPrimeC[PI];
#pragma unroll
    for (int l = 0; l < M; l++) {
        const int h = 1 << (M - 1 - l);
#pragma unroll
        for (int t = 0; t < (1 << M); t++) {
            if (t & h) continue;
            const int e = (t & (h - 1)) * (16 / h);
            const uint32_t a = x[t], b = x[t + h];
            x[t] = ad<PI>(a, b);
            x[t + h] = e ? sh<PI>(a - b + p, c_lines.f[PI][e]) : sb<PI>(a, b);
        }
    }
}

// dft_dif for inputs whose slots t >= NZ are zero (NZ a power of two; the
// caller sets them to the constant 0).  While the half distance h is at
// least NZ a level's partner is zero, so (a, 0) -> (a, a w): the level costs
// only the multiplications of its nonzero slots, and all-zero pairs are
// skipped; once h < NZ every slot is live and the levels are dft_dif's.
template <int PI, int M, int NZ>
FFG_DEV_INLINE void dft_dif_nz(uint32_t (&x)[1 << M]) {
    constexpr uint32_t p = kPrimeC[PI];
#pragma unroll
    for (int l = 0; l < M; l++) {
        const int h = 1 << (M - 1 - l);
#pragma unroll
        for (int t = 0; t < (1 << M); t++) {
            if (t & h) continue;
            const int e = (t & (h - 1)) * (16 / h);
            if (h >= NZ) {
                if ((t & (h - 1)) >= NZ) continue; // both slots still zero
                x[t + h] = e ? sh<PI>(x[t], c_lines.f[PI][e]) : x[t];
            } else {
                const uint32_t a = x[t], b = x[t + h];
                x[t] = ad<PI>(a, b);
                x[t + h] = e ? sh<PI>(a - b + p, c_lines.f[PI][e]) : sb<PI>(a, b);
            }
        }
    }
}

// The inverse: decimation in time, bit-reversed in, natural out, 2^M times
// the inverse DFT.
template <int PI, int M>
FFG_DEV_INLINE void dft_dit(uint32_t (&x)[1 << M]) {
#pragma unroll
    for (int l = 0; l < M; l++) {
        const int h = 1 << l;
#pragma unroll
        for (int t = 0; t < (1 << M); t++) {
            if (t & h) continue;
            const int e = (t & (h - 1)) * (16 / h);
            const uint32_t u = e ? sh<PI>(x[t + h], c_lines.i[PI][e]) : x[t + h];
            x[t + h] = sb<PI>(x[t], u);
            x[t] = ad<PI>(x[t], u);
        }
    }
}

// One radix-2^M step at stride 2^sl over every 2^n block of every line.
// Threads split the 2^(n-M) groups of a block first (consecutive threads,
// consecutive j: conflict-free with the padding for sl = 0 or sl >= 5), and
// the block-lines second; a thread loads its group's twiddles once for all
// the block-lines it handles.
template <int PI, int M, bool DIF, bool TW>
FFG_DEV_INLINE void line_step(uint32_t *__restrict__ s, uint32_t lines_lg, uint32_t nblk, uint32_t n,
                              uint32_t stride, uint32_t sl, const uint2 *__restrict__ tw) {
    constexpr int R = 1 << M;
    const uint32_t np_lg = n - M;
    const uint32_t tp_lg = np_lg < kLineThreadsLg ? np_lg : kLineThreadsLg;
    const uint32_t tp = threadIdx.x & ((1u << tp_lg) - 1), tl = threadIdx.x >> tp_lg;
    const uint32_t lanes = kLineThreads >> tp_lg;
    const uint32_t vlines = nblk << lines_lg, lmask = (1u << lines_lg) - 1;
    const uint32_t S = 1u << sl;
    const uint32_t Sp = S + (S >> 5); // padded distance of t -> t + 1 (sl = 0 or sl >= 5)
    for (uint32_t pos = tp; pos < (1u << np_lg); pos += 1u << tp_lg) {
        const uint32_t j = pos & (S - 1);
        const uint32_t base = ((pos >> sl) << (M + sl)) + j;
        uint2 w[TW ? R - 1 : 1];
        if (TW) {
#pragma unroll
            for (int t = 1; t < R; t++) w[t - 1] = __ldg(&tw[(t - 1) * S + j]);
        }
        for (uint32_t vl = tl; vl < vlines; vl += lanes) {
            uint32_t *L = s + (vl & lmask) * stride + pad_idx(((vl >> lines_lg) << n) + base);
            uint32_t x[R];
#pragma unroll
            for (int t = 0; t < R; t++) x[t] = L[t * Sp];
            if (DIF) {
                dft_dif<PI, M>(x);
                if (TW) {
#pragma unroll
                    for (int t = 1; t < R; t++) x[t] = sh<PI>(x[t], w[t - 1]);
                }
            } else {
                if (TW) {
#pragma unroll
                    for (int t = 1; t < R; t++) x[t] = sh<PI>(x[t], w[t - 1]);
                }
                dft_dit<PI, M>(x);
            }
#pragma unroll
            for (int t = 0; t < R; t++) L[t * Sp] = x[t];
        }
    }
}

// Steps at stride 1 need no twiddles (j = 0); schedule() gives radix 32
// only there, so the twiddled steps hold at most 16 words and 15 twiddles.
// A stride-1 step has the radix of the whole block when n < 6 (the column
// lines of L = 3 2^11 have n = 3).
template <int PI, bool DIF>
FFG_DEV_INLINE void line_step_m(int M, uint32_t *s, uint32_t lines_lg, uint32_t nblk, uint32_t n, uint32_t stride,
                                uint32_t sl, const uint2 *tw) {
    if (sl == 0) {
        switch (M) {
        case 1: line_step<PI, 1, DIF, false>(s, lines_lg, nblk, n, stride, 0, tw); break;
        case 2: line_step<PI, 2, DIF, false>(s, lines_lg, nblk, n, stride, 0, tw); break;
        case 3: line_step<PI, 3, DIF, false>(s, lines_lg, nblk, n, stride, 0, tw); break;
        case 4: line_step<PI, 4, DIF, false>(s, lines_lg, nblk, n, stride, 0, tw); break;
        default: line_step<PI, 5, DIF, false>(s, lines_lg, nblk, n, stride, 0, tw); break;
        }
        return;
    }
    switch (M) {
    case 1: line_step<PI, 1, DIF, true>(s, lines_lg, nblk, n, stride, sl, tw); break;
    case 2: line_step<PI, 2, DIF, true>(s, lines_lg, nblk, n, stride, sl, tw); break;
    case 3: line_step<PI, 3, DIF, true>(s, lines_lg, nblk, n, stride, sl, tw); break;
    default: line_step<PI, 4, DIF, true>(s, lines_lg, nblk, n, stride, sl, tw); break;
    }
}

// Radix-3 DIF step on every line: x_q at j + q 2^n (q = 0, 1, 2) ->
//   y0 = x0 + x1 + x2
//   y1 = (x0 - x2 + ω3 (x1 - x2)) ω_R^j
//   y2 = (x0 - x1 - ω3 (x1 - x2)) ω_R^2j          (ω3^2 = -1 - ω3)
template <int PI>
FFG_DEV_INLINE void r3_dif(uint32_t *s, uint32_t lines_lg, uint32_t n, uint32_t stride, const uint4 *r3f) {
    constexpr uint32_t p = kPrimeC[PI];
    const uint32_t B = 1u << n;
    for (uint32_t g = threadIdx.x; g < (B << lines_lg); g += kLineThreads) {
        const uint32_t j = g & (B - 1);
        uint32_t *L = s + (g >> n) * stride;
        const uint32_t x0 = L[pad_idx(j)], x1 = L[pad_idx(j + B)], x2 = L[pad_idx(j + 2 * B)];
        const uint4 t = __ldg(&r3f[B + j]);
        const uint32_t u = sh<PI>(x1 - x2 + p, c_lines.w3[PI]);
        L[pad_idx(j)] = ad<PI>(ad<PI>(x0, x1), x2);
        L[pad_idx(j + B)] = sh<PI>(ad<PI>(sb<PI>(x0, x2), u), make_uint2(t.x, t.y));
        L[pad_idx(j + 2 * B)] = sh<PI>(sb<PI>(sb<PI>(x0, x1), u), make_uint2(t.z, t.w));
    }
}

// Radix-3 DIT step (inverse of r3_dif up to the factor 3): with
// z1 = y1 ω_R^-j, z2 = y2 ω_R^-2j and ν = ω3^-1,
//   x0 = y0 + z1 + z2,  x1 = y0 - z2 + ν (z1 - z2),  x2 = y0 - z1 - ν (z1 - z2).
template <int PI>
FFG_DEV_INLINE void r3_dit(uint32_t *s, uint32_t lines_lg, uint32_t n, uint32_t stride, const uint4 *r3i) {
    constexpr uint32_t p = kPrimeC[PI];
    const uint32_t B = 1u << n;
    for (uint32_t g = threadIdx.x; g < (B << lines_lg); g += kLineThreads) {
        const uint32_t j = g & (B - 1);
        uint32_t *L = s + (g >> n) * stride;
        const uint4 t = __ldg(&r3i[B + j]);
        const uint32_t y0 = L[pad_idx(j)];
        const uint32_t z1 = sh<PI>(L[pad_idx(j + B)], make_uint2(t.x, t.y));
        const uint32_t z2 = sh<PI>(L[pad_idx(j + 2 * B)], make_uint2(t.z, t.w));
        const uint32_t u = sh<PI>(z1 - z2 + p, c_lines.v3[PI]);
        L[pad_idx(j)] = ad<PI>(ad<PI>(y0, z1), z2);
        L[pad_idx(j + B)] = ad<PI>(sb<PI>(y0, z2), u);
        L[pad_idx(j + 2 * B)] = sb<PI>(sb<PI>(y0, z1), u);
    }
}

// Forward transform of every line (natural order in; position q 2^n + i
// ends holding frequency q + 3 brev_n(i), or brev_n(i) without radix 3).
template <int PI>
FFG_DEV_INLINE void lines_fwd(uint32_t *s, uint32_t lines_lg, uint32_t n, uint32_t r3, uint32_t stride,
                              const PrimeDev &P) {
    if (r3) {
        r3_dif<PI>(s, lines_lg, n, stride, P.r3f);
        __syncthreads();
    }
    int m[4], sl[4];
    const int k = schedule(n, m, sl);
    for (int i = 0; i < k; i++) {
        line_step_m<PI, true>(m[i], s, lines_lg, r3 ? 3 : 1, n, stride, sl[i],
                              P.stw + c_lines.tw_off[sl[i] * 6 + m[i]]);
        __syncthreads();
    }
}

// Inverse transform (digit-reversed in, natural out), unnormalised: the
// result is the line length times the inverse DFT.
template <int PI>
FFG_DEV_INLINE void lines_inv(uint32_t *s, uint32_t lines_lg, uint32_t n, uint32_t r3, uint32_t stride,
                              const PrimeDev &P) {
    int m[4], sl[4];
    const int k = schedule(n, m, sl);
    for (int i = k - 1; i >= 0; i--) {
        line_step_m<PI, false>(m[i], s, lines_lg, r3 ? 3 : 1, n, stride, sl[i],
                               P.istw + c_lines.tw_off[sl[i] * 6 + m[i]]);
        __syncthreads();
    }
    if (r3) {
        r3_dit<PI>(s, lines_lg, n, stride, P.r3i);
        __syncthreads();
    }
}

// ------------------------------------------------------------ tile loads
//
// Loads issue kB accesses per thread before any of them is consumed, so each
// SM keeps tens of kilobytes in flight (Little's law at HBM latency), and
// move 16 bytes per access where the layout allows.

// Rows [0, R) x words [0, 2^wc_lg) of a row-major array g (row stride C
// words, 16-byte aligned rows) into column lines: word (r, c) ->
// smem[c * stride + pad(r)].
template <int kB>
FFG_DEV_INLINE void tile_load(uint32_t *__restrict__ smem, uint32_t stride, const uint32_t *g, uint32_t C, uint32_t R,
                              uint32_t wc_lg) {
    const uint32_t q_lg = wc_lg - 2, qm = (1u << q_lg) - 1; // 16-byte quads per row
    const uint32_t items = R << q_lg;
    for (uint32_t base = threadIdx.x; base < items; base += kLineThreads * kB) {
        uint4 v[kB];
#pragma unroll
        for (int b = 0; b < kB; b++) {
            const uint32_t it = base + b * kLineThreads;
            if (it < items) v[b] = *((const uint4 *)(g + (size_t)(it >> q_lg) * C) + (it & qm));
        }
#pragma unroll
        for (int b = 0; b < kB; b++) {
            const uint32_t it = base + b * kLineThreads;
            if (it < items) {
                uint32_t *d = smem + ((it & qm) << 2) * stride + pad_idx(it >> q_lg);
                d[0] = v[b].x;
                d[stride] = v[b].y;
                d[2 * stride] = v[b].z;
                d[3 * stride] = v[b].w;
            }
        }
    }
}

// One contiguous line of n words (a multiple of 4, 16-byte aligned) into
// shared memory at padded positions.
template <int kB>
FFG_DEV_INLINE void line_load(uint32_t *__restrict__ smem, const uint32_t *g, uint32_t n) {
    const uint32_t items = n >> 2;
    for (uint32_t base = threadIdx.x; base < items; base += kLineThreads * kB) {
        uint4 v[kB];
#pragma unroll
        for (int b = 0; b < kB; b++) {
            const uint32_t it = base + b * kLineThreads;
            if (it < items) v[b] = ((const uint4 *)g)[it];
        }
#pragma unroll
        for (int b = 0; b < kB; b++) {
            const uint32_t it = base + b * kLineThreads;
            if (it < items) {
                const uint32_t i = it << 2;
                smem[pad_idx(i)] = v[b].x;
                smem[pad_idx(i + 1)] = v[b].y;
                smem[pad_idx(i + 2)] = v[b].z;
                smem[pad_idx(i + 3)] = v[b].w;
            }
        }
    }
}

// Digits of a column tile straight from the limbs: coefficient
// i = r C + c0 + c (r < R, c < 2^wc_lg), digit off + i of width w of the
// operand (ns limbs), zero at or past cs, reduced mod p into
// smem[c * stride + pad(r)].  The reference's Src reader
// (src/ntt_kernels.c:29-74) for a whole tile, its limb loads batched.
template <int PI, int kB>
FFG_DEV_INLINE void tile_digits(uint32_t *__restrict__ smem, uint32_t stride, const uint64_t *__restrict__ src,
                                uint64_t ns, uint64_t cs, uint64_t off, uint32_t w, uint32_t C, uint32_t R, uint32_t c0,
                                uint32_t wc_lg, const PrimeDev &P) {
    const uint32_t items = R << wc_lg, cm = (1u << wc_lg) - 1;
    const uint64_t mask = (1ull << w) - 1;
    for (uint32_t base = threadIdx.x; base < items; base += kLineThreads * kB) {
        uint64_t lo[kB], hi[kB];
        uint32_t sh[kB];
#pragma unroll
        for (int b = 0; b < kB; b++) {
            const uint32_t it = base + b * kLineThreads;
            const uint64_t i = (uint64_t)(it >> wc_lg) * C + c0 + (it & cm);
            const uint64_t bit = (off + i) * w, q = bit >> 6;
            sh[b] = (uint32_t)(bit & 63);
            const bool ok = it < items && i < cs;
            lo[b] = ok && q < ns ? __ldg(&src[q]) : 0;
            hi[b] = ok && sh[b] + w > 64 && q + 1 < ns ? __ldg(&src[q + 1]) : 0;
        }
#pragma unroll
        for (int b = 0; b < kB; b++) {
            const uint32_t it = base + b * kLineThreads;
            if (it < items) {
                const uint64_t v = sh[b] ? (lo[b] >> sh[b]) | (hi[b] << (64 - sh[b])) : lo[b];
                smem[(it & cm) * stride + pad_idx(it >> wc_lg)] = reduce_digit(v & mask, P);
            }
        }
    }
}

// ω_L^e (e < L, L | M) in Montgomery form, from the two small tables.
template <int PI>
FFG_DEV_INLINE uint32_t twm(const PrimeDev &P, uint64_t E) {
    const uint32_t lo = __ldg(&P.twl[E & (FFG_TW_LO - 1)]);
    const uint32_t hi = __ldg(&P.twh[E >> FFG_TW_LO_LG]);
    return mo<PI>(lo, hi);
}

} // namespace ffg
