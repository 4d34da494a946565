// The decimal conversion driver: big_to_string (src/decimal.c:229-281) on the
// device, breadth first.  With
// P_l = 10^(19 2^l) of exactly s_l bits and T the least level with
// 2 (s_T - 1) >= bits(x), level l splits every piece x < 2^(2 s_l) into
// q = floor(x / P_l) and r = x mod P_l by Barrett's method
//     q1 = x >> (s - 1),  q = (q1 m) >> (s + 1),  m <= floor(2^(2s) / P)
// (src/decimal.c:76-89), then one correction: k = floor((x - q P) / P) from
// 64-bit windows (k_khat_batch, exact or one too large), r = x - q P - k P,
// q += k (k_comb_batch).  All pieces of a level share each launch: two
// shifts, two batched products (grouped by plan, src/decimal.c:177-203 does
// them one at a time), the estimate and one combination.  Pieces below
// 10^(19 2^(leaf + 1)) become 19 2^(leaf + 1) digits each (k_leaf_digits,
// the reference's dec_leaf, src/decimal.c:139-150); leading zeros are
// dropped on the host.  An estimate out of its range (which the bounds rule
// out) raises a flag and the conversion is redone on the host path.
//
// The powers and their reciprocals depend only on the level; they stay on
// the device between calls.  The reciprocals come from Newton's iteration
// from below (src/decimal.c:39-71 restated so that every sign is known):
//     y' = y + floor(y (2^(2s) - P y) / 2^(2s))  <=  floor(2^(2s) / P),
// started at level l from (m_(l-1))^2 >> (4 s_(l-1) - 2 s_l), two steps a
// level (the error of the start squares twice to a few units).

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "ffg.h"
#include "ffg_hostctx.h"
#include "ffg_internal.h"


namespace ffg {

// Leaves: pieces below 10^(19 2^(kDecLeafLg + 1)) = 10^2432 (at most 128 limbs),
// one thread each.  The reference stops its recursion two levels lower
// (DEC_LEAF_LG = 4, src/decimal.c); here the two lowest levels would hold tens
// of thousands of pieces whose job records cost more host time than their
// arithmetic costs the GPU.
static const int kDecLeafLg = 6;
static const uint64_t kDec19 = 10000000000000000000ull;

typedef unsigned __int128 u128h;

// The decimal host entry points' device copy of their number, kept between calls.
static uint64_t *g_dec_in = nullptr;
static size_t g_dec_in_cap = 0;

struct DecLevel {
    uint64_t *P = nullptr, *m = nullptr; // dedicated allocations (kept between calls)
    uint64_t nP = 0, nm = 0;
    uint64_t s = 0;                      // bits of P
};
static std::vector<DecLevel> g_dec;
static double g_dec_ms = 0; // device time of the last conversion (levels, leaves, zero scan)

static uint64_t limbs_of(uint64_t bits) { return std::max<uint64_t>(1, (bits + 63) / 64); }

// Device helpers on stream st, temporaries from the arena.
static int dev_upload_jobs(const void *h, size_t bytes, void **d, cudaStream_t st) {
    *d = arena_alloc(std::max<size_t>(bytes, 16));
    if (!*d) return fail(FFG_E_NOMEM, "device arena: job records");
    if (bytes) CK(cudaMemcpyAsync(*d, h, bytes, cudaMemcpyHostToDevice, st));
    return FFG_OK;
}

static int dev_shift(std::vector<ShiftJob> &jobs, cudaStream_t st) {
    if (jobs.empty()) return FFG_OK;
    uint64_t mx = 0;
    for (auto &j : jobs) mx = std::max(mx, j.nout);
    void *d;
    int rc = dev_upload_jobs(jobs.data(), jobs.size() * sizeof(ShiftJob), &d, st);
    if (rc) return rc;
    cudaError_t e = launch_shift_batch((const ShiftJob *)d, (uint32_t)jobs.size(), mx, st);
    return e ? fail(FFG_E_CUDA, "decimal shift: %s", cudaGetErrorString(e)) : FFG_OK;
}

static int dev_comb(std::vector<CombJob> &jobs, cudaStream_t st) {
    if (jobs.empty()) return FFG_OK;
    uint64_t mx = 0;
    for (auto &j : jobs) mx = std::max(mx, j.len);
    const uint32_t nl = comb_nl(mx);
    for (auto &j : jobs) {
        j.maps = (uint32_t *)arena_alloc((size_t)comb_ctas(j.len, nl) * 4);
        if (!j.maps) return fail(FFG_E_NOMEM, "device arena: combination maps");
        j.ticket = ticket_get();
    }
    void *d;
    int rc = dev_upload_jobs(jobs.data(), jobs.size() * sizeof(CombJob), &d, st);
    if (rc) return rc;
    cudaError_t e = launch_comb_batch((const CombJob *)d, (uint32_t)jobs.size(), mx, st);
    return e ? fail(FFG_E_CUDA, "decimal combination: %s", cudaGetErrorString(e)) : FFG_OK;
}

// Products out_i = a_i b_i (out_i: na + nb + 1 limbs), the plain thresholds
// (a level's products share one shape: the plan is looked up once a shape).
static int dev_products(std::vector<BJob> &jobs, cudaStream_t st) {
    std::vector<BJob> run;
    run.reserve(jobs.size());
    BJob last{};
    bool have = false;
    for (BJob J : jobs) {
        if (have && J.bits_a == last.bits_a && J.bits_b == last.bits_b && J.square == last.square) {
            J.school = last.school;
            J.pl = last.pl;
        } else {
            const int rc = method_plan(FFG_M_PLAIN, J.bits_a, J.bits_b, J.square, &J);
            if (rc) return rc;
            last = J;
            have = true;
        }
        run.push_back(J);
    }
    return run_batch(run, st);
}

static BJob bjob(const uint64_t *a, uint64_t na, uint64_t ba, const uint64_t *b, uint64_t nb, uint64_t bb, uint64_t *out,
                 bool square) {
    BJob J{};
    J.a = a, J.b = square ? a : b, J.na = na, J.nb = square ? na : nb;
    J.bits_a = std::min(ba, 64 * na), J.bits_b = square ? J.bits_a : std::min(bb, 64 * nb);
    J.out = out, J.square = square;
    return J;
}

static uint32_t top_bits_of(uint64_t bits) { return (uint32_t)(bits & 63); }

// One Newton step from below for m ~ 2^(2s) / P (y: ny limbs, at most s + 1 bits;
// ynew: limbs_of(s + 1)).
static int newton_step(const DecLevel &L, const uint64_t *y, uint64_t ny, uint64_t *ynew, cudaStream_t st) {
    const uint64_t s = L.s, len2 = limbs_of(2 * s);
    uint64_t *d = (uint64_t *)arena_alloc((L.nP + ny + 1) * 8);
    uint64_t *e = (uint64_t *)arena_alloc(len2 * 8);
    uint64_t *u = (uint64_t *)arena_alloc((ny + len2 + 1) * 8);
    uint64_t *w = (uint64_t *)arena_alloc(limbs_of(s + 1) * 8);
    if (!d || !e || !u || !w) return fail(FFG_E_NOMEM, "device arena: Newton step");
    std::vector<BJob> p1{bjob(L.P, L.nP, s, y, ny, s + 1, d, false)};
    int rc = dev_products(p1, st);
    if (rc) return rc;
    // e = 2^(2s) - P y: two's complement over 2s bits (0 < P y < 2^(2s))
    CombJob c{};
    c.src[0] = d, c.n[0] = std::min<uint64_t>(L.nP + ny + 1, len2), c.mul[0] = -1;
    c.out = e, c.len = len2, c.top_bits = top_bits_of(2 * s);
    std::vector<CombJob> cj{c};
    if ((rc = dev_comb(cj, st))) return rc;
    std::vector<BJob> p2{bjob(y, ny, s + 1, e, len2, 2 * s, u, false)};
    if ((rc = dev_products(p2, st))) return rc;
    std::vector<ShiftJob> sj{ShiftJob{u, ny + len2 + 1, w, limbs_of(s + 1), 2 * s}};
    if ((rc = dev_shift(sj, st))) return rc;
    CombJob c2{};
    c2.src[0] = y, c2.n[0] = ny, c2.mul[0] = 1;
    c2.src[1] = w, c2.n[1] = limbs_of(s + 1), c2.mul[1] = 1;
    c2.out = ynew, c2.len = limbs_of(s + 1);
    std::vector<CombJob> cj2{c2};
    return dev_comb(cj2, st);
}

void dec_free() {
    for (auto &L : g_dec) {
        if (L.P) cudaFree(L.P);
        if (L.m) cudaFree(L.m);
    }
    g_dec.clear();
    if (g_dec_in) cudaFree(g_dec_in);
    g_dec_in = nullptr;
    g_dec_in_cap = 0;
}

// Level l (> 0) of the cache from level l - 1: P_l = P_(l-1)^2 with its exact
// bit length, then m_l from (m_(l-1))^2 and two Newton steps.
static int dec_level(int l, cudaStream_t st) {
    DecLevel &L = g_dec[l];
    const DecLevel &B = g_dec[l - 1];
    CK(cudaStreamSynchronize(st));
    arena_reset();
    const uint64_t nsq = 2 * B.nP + 1;
    CK(cudaMalloc(&L.P, nsq * 8));
    std::vector<BJob> sq{bjob(B.P, B.nP, B.s, nullptr, 0, 0, L.P, true)};
    int rc = dev_products(sq, st);
    if (rc) return rc;
    uint64_t *dbits = (uint64_t *)arena_alloc(8);
    if (!dbits) return fail(FFG_E_NOMEM, "device arena: bit length");
    cudaError_t e = launch_bit_length(L.P, nsq, dbits, st);
    if (e) return fail(FFG_E_CUDA, "decimal powers: %s", cudaGetErrorString(e));
    CK(cudaMemcpyAsync(&L.s, dbits, 8, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    L.nP = limbs_of(L.s);
    L.nm = limbs_of(L.s + 1);
    CK(cudaMalloc(&L.m, L.nm * 8));
    uint64_t *sqm = (uint64_t *)arena_alloc((2 * B.nm + 1) * 8);
    uint64_t *y0 = (uint64_t *)arena_alloc(L.nm * 8), *y1 = (uint64_t *)arena_alloc(L.nm * 8);
    if (!sqm || !y0 || !y1) return fail(FFG_E_NOMEM, "device arena: reciprocal");
    std::vector<BJob> msq{bjob(B.m, B.nm, B.s + 1, nullptr, 0, 0, sqm, true)};
    if ((rc = dev_products(msq, st))) return rc;
    std::vector<ShiftJob> sh{ShiftJob{sqm, 2 * B.nm + 1, y0, L.nm, 4 * B.s - 2 * L.s}};
    if ((rc = dev_shift(sh, st))) return rc;
    if ((rc = newton_step(L, y0, L.nm, y1, st))) return rc;
    if ((rc = newton_step(L, y1, L.nm, L.m, st))) return rc;
    CK(cudaStreamSynchronize(st));
    return FFG_OK;
}

// Levels 0..T of powers and reciprocals (kept between calls).
static int dec_prepare(int T, cudaStream_t st) {
    while ((int)g_dec.size() <= T) {
        const int l = (int)g_dec.size();
        DecLevel L;
        if (l == 0) {
            L.s = 64, L.nP = 1, L.nm = 2;
            CK(cudaMalloc(&L.P, 8));
            CK(cudaMalloc(&L.m, 16));
            const uint64_t m0[2] = {(uint64_t)((~(u128h)0) / kDec19), (uint64_t)(((~(u128h)0) / kDec19) >> 64)};
            CK(cudaMemcpy(L.P, &kDec19, 8, cudaMemcpyHostToDevice));
            CK(cudaMemcpy(L.m, m0, 16, cudaMemcpyHostToDevice));
            g_dec.push_back(L);
            continue;
        }
        g_dec.push_back(DecLevel{});
        const int rc = dec_level(l, st);
        if (rc) { // a level left incomplete is not kept
            cudaStreamSynchronize(st);
            if (g_dec.back().P) cudaFree(g_dec.back().P);
            if (g_dec.back().m) cudaFree(g_dec.back().m);
            g_dec.pop_back();
            return rc;
        }
    }
    return FFG_OK;
}

// The conversion proper; *err_flag set on the device when a correction fell
// outside its range (the caller then converts on the host path).
// Where a streamed conversion sends its digits (ffg_to_decimal_stream).
struct DecSink {
    ffg_digit_sink fn;
    void *user;
};

static int dec_leaves_streamed(const LeafJob *dl, uint64_t nleaves, uint32_t chunks, uint64_t v, char *dd,
                               const uint32_t *flags, int T, const DecSink &sink, size_t *nout, bool *fallback,
                               cudaStream_t st);

static int dec_device(const uint64_t *x, uint64_t nx, uint64_t bx, char **out, size_t *nout, bool *fallback,
                      cudaStream_t st, const DecSink *sink = nullptr) {
    *fallback = false;
    int T = 0;
    // powers as needed for the choice of T
    while (true) {
        int rc = dec_prepare(T, st);
        if (rc) return rc;
        if (2 * (g_dec[T].s - 1) >= bx) break;
        T++;
    }
    if (T <= kDecLeafLg + 1) {
        *fallback = true; // small numbers: the host path
        return FFG_OK;
    }
    CK(cudaStreamSynchronize(st));
    arena_reset();
    ev_record(g.ev0, st);
    // flags per level: [2 l] estimate out of range, [2 l + 1] negative remainder
    uint32_t *flags = (uint32_t *)arena_alloc(8 * (T + 1));
    uint64_t *one = (uint64_t *)arena_alloc(8);
    if (!flags || !one) return fail(FFG_E_NOMEM, "device arena: flag");
    CK(cudaMemsetAsync(flags, 0, 8 * (T + 1), st));
    const uint64_t h_one = 1;
    CK(cudaMemcpyAsync(one, &h_one, 8, cudaMemcpyHostToDevice, st));
    // pieces of the current level: pointer, limbs, bit bound
    struct Piece {
        const uint64_t *d;
        uint64_t n, bits;
    };
    std::vector<Piece> cur{Piece{x, nx, bx}};
    for (int l = T; l > kDecLeafLg; l--) {
        const DecLevel &L = g_dec[l];
        const uint64_t s = L.s, cnt = cur.size();
        const uint64_t nq1 = limbs_of(s + 1), nt = nq1 + L.nm + 1, nq = limbs_of(s + 1), nqp = nq + L.nP + 1;
        const uint64_t nr = limbs_of(s + 1), nqo = limbs_of(s + 1);
        uint64_t *q1 = (uint64_t *)arena_alloc(cnt * nq1 * 8), *t = (uint64_t *)arena_alloc(cnt * nt * 8);
        uint64_t *q = (uint64_t *)arena_alloc(cnt * nq * 8), *qp = (uint64_t *)arena_alloc(cnt * nqp * 8);
        uint32_t *kh = (uint32_t *)arena_alloc(cnt * 4), *sg = (uint32_t *)arena_alloc(cnt * 4);
        uint64_t *r1 = (uint64_t *)arena_alloc(cnt * nr * 8);
        uint64_t *r = (uint64_t *)arena_alloc(cnt * nr * 8), *qo = (uint64_t *)arena_alloc(cnt * nqo * 8);
        if (!q1 || !t || !q || !qp || !kh || !sg || !r1 || !r || !qo)
            return fail(FFG_E_NOMEM, "device arena: decimal level %d", l);
        std::vector<ShiftJob> sh;
        std::vector<BJob> pr;
        for (uint64_t p = 0; p < cnt; p++) sh.push_back(ShiftJob{cur[p].d, cur[p].n, q1 + p * nq1, nq1, s - 1});
        int rc = dev_shift(sh, st);
        if (rc) return rc;
        for (uint64_t p = 0; p < cnt; p++)
            pr.push_back(bjob(q1 + p * nq1, nq1, s + 1, L.m, L.nm, s + 1, t + p * nt, false));
        if ((rc = dev_products(pr, st))) return rc;
        sh.clear();
        for (uint64_t p = 0; p < cnt; p++) sh.push_back(ShiftJob{t + p * nt, nt, q + p * nq, nq, s + 1});
        if ((rc = dev_shift(sh, st))) return rc;
        pr.clear();
        for (uint64_t p = 0; p < cnt; p++) pr.push_back(bjob(q + p * nq, nq, s + 1, L.P, L.nP, s, qp + p * nqp, false));
        if ((rc = dev_products(pr, st))) return rc;
        std::vector<KhatJob> kj;
        for (uint64_t p = 0; p < cnt; p++)
            kj.push_back(KhatJob{cur[p].d, qp + p * nqp, L.P, cur[p].n, nqp, L.nP, s, kh + p, flags + 2 * l});
        void *dk;
        if ((rc = dev_upload_jobs(kj.data(), kj.size() * sizeof(KhatJob), &dk, st))) return rc;
        cudaError_t e = launch_khat_batch((const KhatJob *)dk, (uint32_t)cnt, st);
        if (e) return fail(FFG_E_CUDA, "decimal estimate: %s", cudaGetErrorString(e));
        // r1 = x - q P - k P over s + 1 bits (negative when k is one too
        // large: then r1 + P and q + k - 1), its sign per piece
        std::vector<CombJob> cj;
        for (uint64_t p = 0; p < cnt; p++) {
            CombJob c{};
            c.src[0] = cur[p].d, c.n[0] = std::min(cur[p].n, nr), c.mul[0] = 1;
            c.src[1] = qp + p * nqp, c.n[1] = std::min(nqp, nr), c.mul[1] = -1;
            c.src[2] = L.P, c.n[2] = std::min(L.nP, nr), c.mul[2] = -1, c.scale[2] = kh + p;
            c.out = r1 + p * nr, c.len = nr, c.sign_out = sg + p;
            cj.push_back(c);
        }
        if ((rc = dev_comb(cj, st))) return rc;
        cj.clear();
        for (uint64_t p = 0; p < cnt; p++) {
            CombJob c{}; // r = r1 + sign P
            c.src[0] = r1 + p * nr, c.n[0] = nr, c.mul[0] = 1;
            c.src[1] = L.P, c.n[1] = std::min(L.nP, nr), c.mul[1] = 1, c.scale[1] = sg + p;
            c.out = r + p * nr, c.len = nr, c.neg_flag = flags + 2 * l + 1;
            cj.push_back(c);
            CombJob d{}; // q + k - sign
            d.src[0] = q + p * nq, d.n[0] = nq, d.mul[0] = 1, d.add_dev = kh + p;
            d.src[1] = one, d.n[1] = 1, d.mul[1] = -1, d.scale[1] = sg + p;
            d.out = qo + p * nqo, d.len = nqo;
            cj.push_back(d);
        }
        if ((rc = dev_comb(cj, st))) return rc;
        std::vector<Piece> nxt;
        for (uint64_t p = 0; p < cnt; p++) {
            nxt.push_back(Piece{qo + p * nqo, nqo, s});
            nxt.push_back(Piece{r + p * nr, nr, s});
        }
        cur.swap(nxt);
    }
    // leaves: below P_(leaf + 1), 2 << leaf chunks of 19 digits each
    const uint32_t chunks = 2u << kDecLeafLg;
    std::vector<LeafJob> lj;
    for (auto &p : cur) {
        if (p.n > (uint64_t)FFG_LEAF_MAX_LIMBS) return fail(FFG_E_ARG, "decimal leaf of %llu limbs", (unsigned long long)p.n);
        lj.push_back(LeafJob{p.d, p.n});
    }
    const uint64_t total = (uint64_t)lj.size() * chunks * 19;
    char *dd = (char *)arena_alloc(total);
    void *dl;
    int rc = dd ? dev_upload_jobs(lj.data(), lj.size() * sizeof(LeafJob), &dl, st) : fail(FFG_E_NOMEM, "digits");
    if (rc) return rc;
    const uint64_t v = (uint64_t)((~(u128h)0) / kDec19 - ((u128h)1 << 64));
    if (sink) {
        *out = nullptr;
        return dec_leaves_streamed((const LeafJob *)dl, lj.size(), chunks, v, dd, flags, T, *sink, nout, fallback, st);
    }
    cudaError_t e = launch_leaf_digits((const LeafJob *)dl, (uint32_t)lj.size(), chunks, v, dd, st);
    if (e) return fail(FFG_E_CUDA, "decimal leaves: %s", cudaGetErrorString(e));
    // leading zeros found on the device; only the digits cross to the host
    unsigned long long *dfirst = (unsigned long long *)arena_alloc(8);
    if (!dfirst) return fail(FFG_E_NOMEM, "device arena: digits");
    const unsigned long long none = total - 1;
    CK(cudaMemcpyAsync(dfirst, &none, 8, cudaMemcpyHostToDevice, st));
    if ((e = launch_first_nonzero(dd, total, dfirst, st))) return fail(FFG_E_CUDA, "digits: %s", cudaGetErrorString(e));
    ev_record(g.ev1, st);
    unsigned long long first = 0;
    std::vector<uint32_t> hflags(2 * (T + 1));
    CK(cudaMemcpyAsync(&first, dfirst, 8, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(hflags.data(), flags, 8 * (T + 1), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    float ms = 0;
    if (cudaEventElapsedTime(&ms, g.ev0, g.ev1) == cudaSuccess) g_dec_ms = ms;
    for (int l = 0; l <= T; l++)
        if (hflags[2 * l] || hflags[2 * l + 1]) {
            // not an error: the caller converts another way; the reason stays readable
            g.err = "decimal conversion declined at level " + std::to_string(l) +
                    (hflags[2 * l] ? ": quotient estimate out of range" : ": negative remainder");
            *fallback = true;
            return FFG_OK;
        }
    // the digits land in a pooled pinned buffer (one DMA at full speed, no
    // fresh pages to fault in); the caller returns it with ffg_free
    const uint64_t nd = total - first;
    char *h = (char *)pinned_get(nd + 1);
    if (!h) return fail(FFG_E_NOMEM, "host digits");
    e = cudaMemcpyAsync(h, dd + first, nd, cudaMemcpyDeviceToHost, st);
    if (!e) e = cudaStreamSynchronize(st);
    if (e) {
        pinned_release(h);
        return fail(FFG_E_CUDA, "digits download: %s", cudaGetErrorString(e));
    }
    h[nd] = 0;
    *out = h;
    *nout = nd;
    return FFG_OK;
}

// The leaves of a streamed conversion: the conversion's flags are read first
// (a declined conversion emits nothing); then the leaves run in up to eight
// launches, each followed by the copy of its digits into a pooled pinned
// buffer and an event, and the host hands slice k to the sink (leading zeros
// stripped) while the GPU still computes and copies the slices after it.
static int dec_leaves_streamed(const LeafJob *dl, uint64_t nleaves, uint32_t chunks, uint64_t v, char *dd,
                               const uint32_t *flags, int T, const DecSink &sink, size_t *nout, bool *fallback,
                               cudaStream_t st) {
    std::vector<uint32_t> hflags(2 * (T + 1));
    CK(cudaMemcpyAsync(hflags.data(), flags, 8 * (T + 1), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    for (int l = 0; l <= T; l++)
        if (hflags[2 * l] || hflags[2 * l + 1]) {
            g.err = "decimal conversion declined at level " + std::to_string(l) +
                    (hflags[2 * l] ? ": quotient estimate out of range" : ": negative remainder");
            *fallback = true;
            return FFG_OK;
        }
    const uint64_t per = (uint64_t)chunks * 19, total = nleaves * per;
    char *h = (char *)pinned_get(total);
    if (!h) return fail(FFG_E_NOMEM, "host digits");
    struct Guard {
        char *h;
        cudaStream_t st;
        std::vector<cudaEvent_t> ev;
        ~Guard() {
            cudaStreamSynchronize(st);
            for (auto e : ev)
                if (e) cudaEventDestroy(e);
            pinned_release(h);
        }
    } gd{h, st, {}};
    const uint64_t K = nleaves < 8 ? nleaves : 8;
    std::vector<uint64_t> cut(K + 1);
    for (uint64_t k = 0; k <= K; k++) cut[k] = nleaves * k / K;
    gd.ev.assign(K, nullptr);
    for (uint64_t k = 0; k < K; k++) {
        CK(cudaEventCreateWithFlags(&gd.ev[k], cudaEventDisableTiming));
        const uint64_t j0 = cut[k], n = cut[k + 1] - cut[k];
        cudaError_t e = launch_leaf_digits(dl + j0, (uint32_t)n, chunks, v, dd + j0 * per, st);
        if (e) return fail(FFG_E_CUDA, "decimal leaves: %s", cudaGetErrorString(e));
        CK(cudaMemcpyAsync(h + j0 * per, dd + j0 * per, n * per, cudaMemcpyDeviceToHost, st));
        CK(cudaEventRecord(gd.ev[k], st));
    }
    ev_record(g.ev1, st);
    size_t emitted = 0;
    bool started = false;
    for (uint64_t k = 0; k < K; k++) {
        CK(cudaEventSynchronize(gd.ev[k]));
        const char *p = h + cut[k] * per;
        uint64_t n = (cut[k + 1] - cut[k]) * per;
        if (!started) {
            // the number is nonzero: its first digit is in some slice, and the
            // slices of leading zeros before it emit nothing
            uint64_t z = 0;
            while (z < n && p[z] == '0') z++;
            p += z, n -= z;
            started = n > 0;
        }
        if (n) sink.fn(p, (size_t)n, sink.user);
        emitted += (size_t)n;
    }
    float ms = 0;
    if (cudaEventElapsedTime(&ms, g.ev0, g.ev1) == cudaSuccess) g_dec_ms = ms;
    *nout = emitted;
    return FFG_OK;
}

} // namespace ffg

using namespace ffg;

// Decimal digits of the device number x (nx limbs) into a malloc'd string
// (*out, *nout digits, NUL-terminated); *done 0 when the device path declined
// (small numbers, or a correction out of range) and the caller must convert
// on the host.
extern "C" int ffg_to_decimal_device(const uint64_t *x, size_t nx, char **out, size_t *nout, int *done) {
    std::lock_guard<std::recursive_mutex> lk(g_mu);
    int rc = ensure_ready();
    if (rc) return rc;
    if (!x || !out || !nout || !done) return fail(FFG_E_ARG, "ffg_to_decimal_device arguments");
    cudaStream_t st = g.stream;
    CK(cudaStreamSynchronize(st));
    arena_reset();
    uint64_t *dbits = (uint64_t *)arena_alloc(8), bx = 0;
    if (!dbits) return fail(FFG_E_NOMEM, "device arena: bit length");
    cudaError_t e = launch_bit_length(x, nx, dbits, st);
    if (e) return fail(FFG_E_CUDA, "bit length: %s", cudaGetErrorString(e));
    CK(cudaMemcpyAsync(&bx, dbits, 8, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    bool fallback = false;
    *done = 0;
    if (bx == 0) return FFG_OK;
    rc = dec_device(x, limbs_of(bx), bx, out, nout, &fallback, st);
    if (rc) return rc;
    *done = fallback ? 0 : 1;
    return FFG_OK;
}

extern "C" int ffg_to_decimal_host(const uint64_t *x, size_t nx, char **out, size_t *nout, int *done) {
    std::lock_guard<std::recursive_mutex> lk(g_mu);
    int rc = ensure_ready();
    if (rc) return rc;
    if (!x || !out || !nout || !done) return fail(FFG_E_ARG, "ffg_to_decimal_host arguments");
    while (nx > 1 && x[nx - 1] == 0) nx--;
    *done = 0;
    if (nx == 1 && x[0] == 0) return FFG_OK;
    CK(cudaStreamSynchronize(g.stream));
    arena_reset();
    // the number gets a buffer of its own, kept between calls (dec_device
    // resets the arena), filled through a pinned staging copy
    if (g_dec_in_cap < nx) {
        if (g_dec_in) cudaFree(g_dec_in);
        g_dec_in = nullptr;
        g_dec_in_cap = 0;
        CK(cudaMalloc(&g_dec_in, nx * 8));
        g_dec_in_cap = nx;
    }
    uint64_t *stage = (uint64_t *)pinned_get(nx * 8);
    if (!stage) return fail(FFG_E_NOMEM, "pinned staging: %zu bytes", nx * 8);
    memcpy(stage, x, nx * 8);
    cudaError_t e = cudaMemcpyAsync(g_dec_in, stage, nx * 8, cudaMemcpyHostToDevice, g.stream);
    if (e) {
        cudaStreamSynchronize(g.stream);
        pinned_release(stage);
        return fail(FFG_E_CUDA, "decimal upload: %s", cudaGetErrorString(e));
    }
    rc = ffg_to_decimal_device(g_dec_in, nx, out, nout, done); // synchronizes before returning
    cudaStreamSynchronize(g.stream);
    pinned_release(stage);
    return rc;
}

extern "C" int ffg_to_decimal_stream(const uint64_t *x, size_t nx, ffg_digit_sink sink, void *user, size_t *ndigits,
                                     int *done) {
    std::lock_guard<std::recursive_mutex> lk(g_mu);
    int rc = ensure_ready();
    if (rc) return rc;
    if (!x || !sink || !ndigits || !done) return fail(FFG_E_ARG, "ffg_to_decimal_stream arguments");
    while (nx > 1 && x[nx - 1] == 0) nx--;
    *done = 0;
    *ndigits = 0;
    if (nx == 1 && x[0] == 0) return FFG_OK;
    cudaStream_t st = g.stream;
    CK(cudaStreamSynchronize(st));
    arena_reset();
    // the number gets the conversion's own buffer, kept between calls
    if (g_dec_in_cap < nx) {
        if (g_dec_in) cudaFree(g_dec_in);
        g_dec_in = nullptr;
        g_dec_in_cap = 0;
        CK(cudaMalloc(&g_dec_in, nx * 8));
        g_dec_in_cap = nx;
    }
    uint64_t *stage = (uint64_t *)pinned_get(nx * 8);
    if (!stage) return fail(FFG_E_NOMEM, "pinned staging: %zu bytes", nx * 8);
    memcpy(stage, x, nx * 8);
    cudaError_t e = cudaMemcpyAsync(g_dec_in, stage, nx * 8, cudaMemcpyHostToDevice, st);
    if (!e) e = cudaStreamSynchronize(st);
    pinned_release(stage);
    if (e) return fail(FFG_E_CUDA, "decimal upload: %s", cudaGetErrorString(e));
    uint64_t *dbits = (uint64_t *)arena_alloc(8), bx = 0;
    if (!dbits) return fail(FFG_E_NOMEM, "device arena: bit length");
    if ((e = launch_bit_length(g_dec_in, nx, dbits, st))) return fail(FFG_E_CUDA, "bit length: %s", cudaGetErrorString(e));
    CK(cudaMemcpyAsync(&bx, dbits, 8, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (bx == 0) return FFG_OK;
    bool fallback = false;
    char *unused = nullptr;
    const DecSink ds{sink, user};
    rc = dec_device(g_dec_in, limbs_of(bx), bx, &unused, ndigits, &fallback, st, &ds);
    if (rc) return rc;
    *done = fallback ? 0 : 1;
    return FFG_OK;
}

extern "C" double ffg_last_decimal_ms(void) { return g_dec_ms; }

extern "C" void ffg_decimal_cache_clear(void) {
    std::lock_guard<std::recursive_mutex> lk(g_mu);
    if (g.ready) cudaStreamSynchronize(g.stream);
    dec_free();
}
