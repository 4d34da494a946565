// Host side of the B200 layer: device tables, a block arena, the product
// plan (the reference's width / length choice plus the GPU geometry), the
// multiply orchestration, the device fast-doubling chain, and the C ABI
// declared in include/ffg.h.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <thread>
#include <string>
#include <map>
#include <tuple>
#include <vector>

#include "ffg.h"
#include "ffg_hostctx.h"
#include "ffg_internal.h"

namespace ffg {

typedef unsigned __int128 u128h;

static const uint32_t kP[3] = {2113929217u, 2013265921u, 1811939329u}; // src/ntt_arith.c:48-52
static const uint32_t kG[3] = {5u, 31u, 13u};
static int kMaxLg = 25; // NTT_MAX_LG (src/common.h:46-48); ffg_set_max_lg lowers it like -DNTT_MAX_LG
static const uint32_t kSmallMaxL = 4096;  // one-CTA transform up to this length for a single product
static const int kR3TabLg = 13;           // radix-3 tables cover R = 3 2^n, n < 13
// Doubling steps whose operands have at most this many limbs square by
// schoolbook (k_school_sq_pair, one launch for the pair) instead of the NTT
// (transform + CRT): at these sizes both are latency-bound.  Measured on the
// F(10^8) chain: 256 limbs 0.947 ms, 512 0.939, 768 0.939 (and 8 us less
// than 256 on chains of n ~ 10^5).
static const uint64_t kChainSchoolLimbs = 768;

// ------------------------------------------------------------ host modmath

static uint32_t powmod(uint32_t a, uint64_t e, uint32_t p) {
    uint64_t r = 1, x = a % p;
    for (; e; e >>= 1, x = x * x % p)
        if (e & 1) r = r * x % p;
    return (uint32_t)r;
}
static uint32_t inv_mod(uint32_t a, uint32_t p) { return powmod(a, p - 2, p); }
static uint32_t shoup_q(uint32_t w, uint32_t p) { return (uint32_t)(((uint64_t)w << 32) / p); }
static uint32_t to_mont(uint32_t x, uint32_t p) { return (uint32_t)(((uint64_t)x << 32) % p); }
static uint32_t mulm(uint32_t a, uint32_t b, uint32_t p) { return (uint32_t)((uint64_t)a * b % p); }

GarnerConst garner_const() {
    GarnerConst K;
    for (int i = 0; i < 3; i++) K.p[i] = kP[i];
    K.i12 = inv_mod(kP[0] % kP[1], kP[1]);
    K.i12s = shoup_q(K.i12, kP[1]);
    K.i13 = inv_mod(kP[0] % kP[2], kP[2]);
    K.i13s = shoup_q(K.i13, kP[2]);
    K.i23 = inv_mod(kP[1] % kP[2], kP[2]);
    K.i23s = shoup_q(K.i23, kP[2]);
    K.p12 = (uint64_t)kP[0] * kP[1];
    return K;
}

// ------------------------------------------------------------------ context

Ctx g;
std::recursive_mutex g_mu;

// ------------------------------------------------------------ ticket pool

// Zero words for the in-launch carry settle (see ticket_get in
// ffg_internal.h): the live region is handed out round-robin, captured
// launches take words of the capture region (a cached graph keeps its words
// while later work cycles through the live region), and the last word
// belongs to the allocation-free multiply.
constexpr uint32_t kTicketsLive = 1u << 16, kTicketsCapture = 1u << 13;
static uint32_t *g_tickets = nullptr;
static uint32_t g_ticket_live = 0, g_ticket_cap = 0;
bool g_capturing = false;

uint32_t *ticket_get() {
    if (g_capturing) return g_tickets + kTicketsLive + (g_ticket_cap++ % kTicketsCapture);
    return g_tickets + (g_ticket_live++ % kTicketsLive);
}

static uint32_t *ticket_get_reserved() { return g_tickets + kTicketsLive + kTicketsCapture; }

// ------------------------------------------------------------ profiling

// Launch counter (always on) and, when enabled, CUDA-event brackets around
// every launch of each kernel family, on the stream the kernel runs on.
struct ProfPair {
    int kind;
    cudaEvent_t a, b;
    double bytes;
};
static uint64_t g_launches = 0;
static bool g_prof_on = false;
static uint32_t g_prof_mask = 0;
static std::vector<ProfPair> g_prof_open;
static std::vector<cudaEvent_t> g_ev_pool;
static double g_prof_ms[PK_COUNT], g_prof_bytes[PK_COUNT];
static uint64_t g_prof_n[PK_COUNT];

static cudaEvent_t ev_get() {
    if (!g_ev_pool.empty()) {
        cudaEvent_t e = g_ev_pool.back();
        g_ev_pool.pop_back();
        return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
}

// Inside a stream capture an event becomes a timing node of the graph only
// when recorded as external.
void ev_record(cudaEvent_t e, cudaStream_t st) {
    if (g_capturing) cudaEventRecordWithFlags(e, st, cudaEventRecordExternal);
    else cudaEventRecord(e, st);
}

void prof_begin(int kind, cudaStream_t st) {
    g_launches++;
    if (!g_prof_on || !((g_prof_mask >> kind) & 1)) return;
    ProfPair pp{kind, ev_get(), nullptr, 0};
    ev_record(pp.a, st);
    g_prof_open.push_back(pp);
}

void prof_end(int kind, cudaStream_t st, double bytes) {
    if (!g_prof_on || !((g_prof_mask >> kind) & 1)) return;
    if (g_prof_open.empty() || g_prof_open.back().kind != kind || g_prof_open.back().b) return;
    ProfPair &pp = g_prof_open.back();
    pp.b = ev_get();
    pp.bytes = bytes;
    ev_record(pp.b, st);
}

// Folds finished brackets into the totals (synchronizes on their events).
static void prof_collect() {
    for (auto &pp : g_prof_open) {
        if (pp.b) {
            float ms = 0;
            cudaEventSynchronize(pp.b);
            cudaEventElapsedTime(&ms, pp.a, pp.b);
            g_prof_ms[pp.kind] += ms;
            g_prof_bytes[pp.kind] += pp.bytes;
            g_prof_n[pp.kind]++;
            g_ev_pool.push_back(pp.b);
        }
        g_ev_pool.push_back(pp.a);
    }
    g_prof_open.clear();
}

int fail(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g.err = buf;
    return code;
}

// Every (stride 2^sl, radix 2^M) step a transform of up to 2^FFG_LINE_LG
// words can take, with sl > 0 (steps at stride 1 need no twiddles): the line
// schedules and the fixed-shape row and column kernels pick among them.
// Returns the table's length; off[sl * 6 + M] is each step's offset.
static size_t step_table_layout(uint32_t *off) {
    for (int k = 0; k < 15 * 6; k++) off[k] = ~0u;
    size_t total = 0;
    for (int sl = 1; sl < FFG_LINE_LG; sl++)
        for (int M = 1; M <= 5 && sl + M <= FFG_LINE_LG; M++) {
            off[sl * 6 + M] = (uint32_t)total;
            total += (((size_t)1 << M) - 1) << sl;
        }
    return total;
}

static uint32_t brev_bits(uint32_t x, int bits) {
    uint32_t r = 0;
    for (int b = 0; b < bits; b++) r |= ((x >> b) & 1u) << (bits - 1 - b);
    return r;
}

// Device tables for the three primes (see PrimeDev) and the constant-memory
// roots of the line transforms (LineConsts).
static int build_tables() {
    LineConsts lc{};
    const size_t nstw = step_table_layout(lc.tw_off), nr3 = (size_t)1 << kR3TabLg;
    const size_t ntwh = (size_t)(FFG_M / FFG_TW_LO);
    const size_t per = nstw * 2 * sizeof(uint2) + nr3 * 2 * sizeof(uint4) + (FFG_TW_LO + ntwh) * sizeof(uint32_t);
    std::vector<char> host(per * 3);
    CK(cudaMalloc(&g.tables, per * 3));
    if (!g_tickets) {
        const size_t nt = (size_t)kTicketsLive + kTicketsCapture + 1;
        CK(cudaMalloc(&g_tickets, nt * sizeof(uint32_t)));
        CK(cudaMemset(g_tickets, 0, nt * sizeof(uint32_t)));
    }
    for (int k = 0; k < 3; k++) {
        const uint32_t p = kP[k], gen = kG[k];
        char *hb = host.data() + per * k;
        char *db = (char *)g.tables + per * k;
        uint2 *stw = (uint2 *)hb, *istw = stw + nstw;
        uint4 *r3f = (uint4 *)(istw + nstw), *r3i = r3f + nr3;
        uint32_t *twl = (uint32_t *)(r3i + nr3), *twh = twl + FFG_TW_LO;
        // step twiddles: slot t of group j at stride S = 2^sl, radix 2^M gets
        // ω_N^(j brev_M(t)), N = 2^M S, at (t - 1) S + j
        for (int sl = 1; sl < 15; sl++)
            for (int M = 1; M <= 5; M++) {
                const uint32_t o = lc.tw_off[sl * 6 + M];
                if (o == ~0u) continue;
                const uint64_t S = (uint64_t)1 << sl, N = S << M;
                const uint32_t wN = powmod(gen, (p - 1) / N, p), wNi = inv_mod(wN, p);
                for (uint32_t t = 1; t < (1u << M); t++) {
                    const uint32_t e = brev_bits(t, M);
                    const uint32_t a = powmod(wN, e, p), ai = powmod(wNi, e, p);
                    uint32_t c = 1, ci = 1;
                    for (uint64_t j = 0; j < S; j++) {
                        stw[o + (t - 1) * S + j] = make_uint2(c, shoup_q(c, p));
                        istw[o + (t - 1) * S + j] = make_uint2(ci, shoup_q(ci, p));
                        c = mulm(c, a, p);
                        ci = mulm(ci, ai, p);
                    }
                }
            }
        r3f[0] = r3i[0] = make_uint4(0, 0, 0, 0);
        for (int n = 0; n < kR3TabLg; n++) {
            const uint64_t B = (uint64_t)1 << n, R = 3 * B;
            uint32_t w = powmod(gen, (p - 1) / R, p), wi = inv_mod(w, p);
            uint32_t c = 1, ci = 1;
            for (uint64_t j = 0; j < B; j++) {
                uint32_t c2 = mulm(c, c, p), ci2 = mulm(ci, ci, p);
                r3f[B + j] = make_uint4(c, shoup_q(c, p), c2, shoup_q(c2, p));
                r3i[B + j] = make_uint4(ci, shoup_q(ci, p), ci2, shoup_q(ci2, p));
                c = mulm(c, w, p);
                ci = mulm(ci, wi, p);
            }
        }
        const uint32_t wM = powmod(gen, (p - 1) / FFG_M, p), wMh = powmod(wM, FFG_TW_LO, p);
        uint32_t c = 1;
        for (uint32_t e = 0; e < FFG_TW_LO; e++, c = mulm(c, wM, p)) twl[e] = to_mont(c, p);
        c = 1;
        for (size_t e = 0; e < ntwh; e++, c = mulm(c, wMh, p)) twh[e] = to_mont(c, p);

        PrimeDev &P = g.P3.pr[k];
        P.p = p;
        uint32_t inv = p; // p^-1 mod 2^32 by Newton (p odd): 3 -> 6 -> 12 -> 24 -> 48 bits
        for (int it = 0; it < 4; it++) inv *= 2 - p * inv;
        P.pinv = inv;
        P.w3 = powmod(gen, (p - 1) / 3, p);
        P.w3s = shoup_q(P.w3, p);
        P.v3 = inv_mod(P.w3, p);
        P.v3s = shoup_q(P.v3, p);
        P.c32 = (uint32_t)((1ull << 32) % p);
        P.c32s = shoup_q(P.c32, p);
        P.stw = (const uint2 *)db;
        P.istw = P.stw + nstw;
        P.r3f = (const uint4 *)(P.istw + nstw);
        P.r3i = P.r3f + nr3;
        P.twl = (const uint32_t *)(P.r3i + nr3);
        P.twh = P.twl + FFG_TW_LO;

        const uint32_t w32 = powmod(gen, (p - 1) / 32, p), w32i = inv_mod(w32, p);
        uint32_t f = 1, fi = 1;
        for (int e = 0; e < 16; e++) {
            lc.f[k][e] = make_uint2(f, shoup_q(f, p));
            lc.i[k][e] = make_uint2(fi, shoup_q(fi, p));
            f = mulm(f, w32, p);
            fi = mulm(fi, w32i, p);
        }
        lc.w3[k] = make_uint2(P.w3, P.w3s);
        lc.v3[k] = make_uint2(P.v3, P.v3s);
        lc.pinv[k] = P.pinv;
    }
    CK(cudaMemcpy(g.tables, host.data(), per * 3, cudaMemcpyHostToDevice));
    CK(set_line_consts(lc));
    CK(set_line_consts_rows(lc));
    CK(set_line_consts_cols(lc));
    return FFG_OK;
}

int ensure_ready() {
    if (g.ready) {
        if (g.device >= 0) CK(cudaSetDevice(g.device));
        return FFG_OK;
    }
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return fail(FFG_E_NODEV, "no CUDA device");
    if (g.device >= 0) CK(cudaSetDevice(g.device));
    else CK(cudaGetDevice(&g.device)); // the device this context is created on
    CK(cudaStreamCreateWithFlags(&g.stream, cudaStreamNonBlocking));
    CK(cudaEventCreate(&g.ev0));
    CK(cudaEventCreate(&g.ev1));
    int rc = build_tables();
    if (rc) return rc;
    g.ready = true;
    return FFG_OK;
}

// -------------------------------------------------------------------- arena

// Bump allocation out of a list of device blocks; blocks are never moved
// while work may be in flight, and reset() (after a synchronize) recycles them.
void arena_reset() {
    for (auto &b : g.blocks) b.used = 0;
}

// g_capturing is set while a stream capture is open: the arena must not grow
// then (no cudaMalloc may be issued); a request that would need a new block
// fails and the capture is abandoned.

void *arena_alloc(size_t bytes) {
    bytes = (bytes + 255) & ~(size_t)255;
    for (auto &b : g.blocks)
        if (b.cap - b.used >= bytes) {
            void *p = b.ptr + b.used;
            b.used += bytes;
            return p;
        }
    if (g_capturing) return nullptr;
    size_t last = g.blocks.empty() ? 0 : g.blocks.back().cap;
    size_t cap = std::max(bytes, std::max((size_t)64 << 20, 2 * last));
    char *p = nullptr;
    if (cudaMalloc(&p, cap) != cudaSuccess) {
        cudaGetLastError();
        cap = bytes;
        if (cudaMalloc(&p, cap) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
    }
    g.blocks.push_back({p, cap, bytes});
    return p;
}

#define ALLOC(var, type, count)                                                                        \
    type *var = (type *)arena_alloc((size_t)(count) * sizeof(type));                                   \
    if (!var) return fail(FFG_E_NOMEM, "device arena: out of memory (%zu bytes)", (size_t)(count) * sizeof(type));

// --------------------------------------------------------------------- plan

// ntt_width_ok (src/mul_ntt.c:55-59)
static bool width_ok(uint64_t bits_a, uint64_t bits_b, unsigned w) {
    const u128h M = (u128h)kP[0] * kP[1] * kP[2];
    uint64_t ca = (bits_a + w - 1) / w, cb = (bits_b + w - 1) / w;
    return ((u128h)(ca < cb ? ca : cb) << (2 * w)) < M;
}

// ntt_length (src/mul_ntt.c:78-93)
uint64_t ntt_length(uint64_t conv, uint32_t *lg_out, uint32_t *r3_out) {
    uint64_t L = 16;
    uint32_t lg = 4, r3 = 0;
    while (L < conv) {
        L <<= 1;
        lg++;
    }
    if (L / 4 * 3 >= conv && L / 4 >= 16) {
        L = L / 4 * 3;
        lg -= 2;
        r3 = 1;
    }
    *lg_out = lg;
    *r3_out = r3;
    return L;
}

// Tuned four-step geometry per transform length 2^lg / 3 2^lg
// (ffg_set_geometry, from the autotuner): row length 2^c and column-tile
// width wc; unset entries follow the default rule below.
Geo g_geo[32][2];

// Shared memory of a four-step column tile (words) and row pass must fit one
// CTA; the radix-3 tables cover column lines 3 2^n with n < kR3TabLg.
bool geo_valid(uint32_t lg, uint32_t r3, uint32_t c, uint32_t wc) {
    if (c < 4 || c > 13 || c > lg || wc < 8 || wc > 64 || (wc & (wc - 1)) || wc > (1u << c)) return false;
    const uint32_t rn = lg - c;
    if (rn < 2 || rn > (r3 ? (uint32_t)kR3TabLg - 1 : (uint32_t)FFG_LINE_LG)) return false;
    const uint32_t R = (r3 ? 3u : 1u) << rn;
    return (size_t)line_stride(R) * wc * 4 <= 200 * 1024;
}

void gpu_geometry(ffg_plan *pl) {
    const Geo &t = g_geo[pl->lg & 31][pl->r3 ? 1 : 0];
    const bool tuned = t.set && geo_valid(pl->lg, pl->r3, t.c, t.wc);
    // short lengths run the one-CTA transform, unless the autotuner measured
    // a four-step geometry faster for this length (a single product or a
    // doubling step's pair gives the one-CTA kernel only six CTAs)
    if (pl->L <= kSmallMaxL && !pl->split && !tuned) {
        pl->kernel = 0;
        pl->row_lg = 0;
        return;
    }
    if (tuned) {
        pl->kernel = 1;
        pl->row_lg = t.c;
        return;
    }
    // rows of 2^c and columns of at least 4: the split's pieces reach down to
    // L = 16 when the transform cap is small (src/mul_split.c:160-161)
    int c = (int)pl->lg - 7;
    c = c < 8 ? 8 : (c > 13 ? 13 : c);
    if (c > (int)pl->lg - 2) c = (int)pl->lg - 2;
    pl->kernel = 1;
    pl->row_lg = (uint32_t)c;
}

// The split's width and piece length (src/mul_split.c:150-177): the widest
// width the CRT bound allows, then the piece length 2^lg over the last five
// lengths by the reference's cost model (tr lg + 5 pairs) 2^lg.
static void split_plan(uint64_t bits_a, uint64_t bits_b, int square, ffg_plan *pl) {
    unsigned bw = 35;
    while (bw > 8 && !width_ok(bits_a, bits_b, bw)) bw--;
    size_t cap = g.max_L < ((size_t)1 << kMaxLg) ? g.max_L : ((size_t)1 << kMaxLg);
    if (cap < 16) cap = 16;
    int lgmax = __builtin_ctzll(cap), lgp = lgmax;
    double best = 0;
    for (int lg = lgmax; lg >= lgmax - 4 && lg >= 10; lg--) {
        uint64_t h = (uint64_t)1 << (lg - 1);
        uint64_t ka = ((bits_a + bw - 1) / bw + h - 1) / h, kb = ((bits_b + bw - 1) / bw + h - 1) / h;
        double ca = (double)ka, cb = (double)kb;
        double tr = square ? 3 * ca - 1 : 2 * (ca + cb) - 1, pairs = square ? ca * (ca + 1) / 2 : ca * cb;
        double cost = (tr * lg + 5 * pairs) * (double)((uint64_t)1 << lg);
        if (lg == lgmax || cost < best) best = cost, lgp = lg;
    }
    const uint64_t Lp = (uint64_t)1 << lgp, H = Lp / 2;
    memset(pl, 0, sizeof *pl);
    pl->split = 1;
    pl->width = bw;
    pl->lg = (uint32_t)lgp;
    pl->L = Lp;
    pl->ca = (bits_a + bw - 1) / bw;
    pl->cb = (bits_b + bw - 1) / bw;
    pl->ka = (pl->ca + H - 1) / H;
    pl->kb = square ? pl->ka : (pl->cb + H - 1) / H;
    pl->conv = pl->ca + pl->cb - 1;
    pl->Lbig = (pl->ka + pl->kb) * H;
}

int plan_select(uint64_t bits_a, uint64_t bits_b, int square, ffg_plan *pl) {
    memset(pl, 0, sizeof *pl);
    uint64_t L = 0;
    for (unsigned w = 32; w <= 35; w++) {
        if (!width_ok(bits_a, bits_b, w)) break;
        uint64_t ca = (bits_a + w - 1) / w, cb = (bits_b + w - 1) / w;
        uint32_t lg, r3;
        uint64_t Lw = ntt_length(ca + cb - 1, &lg, &r3);
        if (L == 0 || Lw < L) {
            L = Lw;
            pl->L = Lw, pl->lg = lg, pl->r3 = r3, pl->width = w;
            pl->ca = ca, pl->cb = cb, pl->conv = ca + cb - 1;
        }
    }
    if (L == 0 || L > g.max_L) split_plan(bits_a, bits_b, square, pl);
    gpu_geometry(pl);
    return FFG_OK;
}

// 2^32 / L mod p as Shoup pairs (undoes the pointwise 2^-32 and the inverse's L).
void scale_consts(uint64_t L, uint32_t *scl, uint32_t *scls) {
    for (int k = 0; k < 3; k++) {
        uint32_t p = kP[k];
        uint32_t v = mulm((uint32_t)((1ull << 32) % p), inv_mod((uint32_t)(L % p), p), p);
        scl[k] = v;
        scls[k] = shoup_q(v, p);
    }
}

// ---------------------------------------------------------------- multiply

FourStep four_step_geometry(const ffg_plan &pl, bool square) {
    FourStep G{};
    G.L = pl.L;
    G.c = pl.row_lg;
    G.rn = pl.lg - G.c;
    G.r3 = pl.r3;
    G.R = (pl.r3 ? 3u : 1u) << G.rn;
    uint32_t wc = 16384u / G.R; // a column tile of about 64 KB of shared memory
    wc = wc < 8 ? 8 : (wc > 64 ? 64 : wc);
    while (wc & (wc - 1)) wc &= wc - 1;
    if (wc > (1u << G.c)) wc = 1u << G.c;
    const Geo &t = g_geo[pl.lg & 31][pl.r3 ? 1 : 0];
    if (t.set && t.c == G.c && geo_valid(pl.lg, pl.r3, t.c, t.wc)) wc = t.wc;
    G.wc = wc;
    G.wc_lg = (uint32_t)__builtin_ctz(wc);
    G.col_stride = line_stride(G.R);
    G.square = square;
    G.mode = ROW_CONV;
    G.mstep = FFG_M / pl.L;
    scale_consts(pl.L, G.scl, G.scls);
    return G;
}

// Products that share one plan (same width, length, squareness), run as one
// batch of transforms, then one CRT each.
// A doubling step's linear pass fused into the CRT of its two squarings
// (k_crt_lin): out_k = alpha_k s1 + beta_k s2 + gamma_k over len limbs.
struct LinFuse {
    uint64_t *out[2];
    uint64_t len;
    int32_t alpha[2], beta[2];
    int64_t gamma[2];
};

static int run_products(const Prod *pr, int count, const ffg_plan &pl, bool square, cudaStream_t st,
                        const LinFuse *fuse = nullptr) {
    const uint64_t L = pl.L;
    uint32_t scl[3], scls[3];
    scale_consts(L, scl, scls);
    std::vector<uint32_t *> ya(count), yb(count);
    for (int i = 0; i < count; i++) {
        ya[i] = (uint32_t *)arena_alloc(3 * L * sizeof(uint32_t));
        yb[i] = square ? nullptr : (uint32_t *)arena_alloc(3 * L * sizeof(uint32_t));
        if (!ya[i] || (!square && !yb[i])) return fail(FFG_E_NOMEM, "device arena: residues of L=%llu",
                                                      (unsigned long long)L);
    }
    const uint32_t w = pl.width;
    cudaError_t e = cudaSuccess;
    double bytes = 0;
    if (count > FFG_CONV_JOBS) return fail(FFG_E_ARG, "%d products in one launch", count);
    if (pl.kernel == 0) {
        ConvJobs jobs{};
        for (int i = 0; i < count; i++) {
            ConvJob &J = jobs.j[i];
            J.a = pr[i].a, J.b = square ? pr[i].a : pr[i].b;
            J.na = pr[i].na, J.nb = square ? pr[i].na : pr[i].nb;
            J.ca = (pr[i].bits_a + w - 1) / w;
            J.cb = square ? J.ca : (pr[i].bits_b + w - 1) / w;
            J.y = ya[i];
            J.y_stride = L;
            J.L_words = (uint32_t)L;
            J.n = pl.lg, J.r3 = pl.r3, J.width = w, J.square = square;
            J.conv = (uint32_t)(J.ca + J.cb - 1);
            memcpy(J.scl, scl, sizeof scl);
            memcpy(J.scls, scls, sizeof scls);
            bytes += 8.0 * (double)(J.na + (square ? 0 : J.nb)) + 12.0 * (double)J.conv;
        }
        e = launch_conv_small(g.P3, jobs, (uint32_t)count, (uint32_t)L, !square, st, bytes);
        if (e) return fail(FFG_E_CUDA, "conv_small: %s", cudaGetErrorString(e));
    } else {
        FourStep G = four_step_geometry(pl, square);
        FSJobs jobs{};
        for (int i = 0; i < count; i++) {
            FSJob &J = jobs.j[i];
            J.a = pr[i].a, J.b = square ? pr[i].a : pr[i].b;
            J.na = pr[i].na, J.nb = square ? pr[i].na : pr[i].nb;
            J.ca = (pr[i].bits_a + w - 1) / w;
            J.cb = square ? J.ca : (pr[i].bits_b + w - 1) / w;
            J.ya = ya[i], J.yb = yb[i];
            J.width = w;
        }
        double limb_bytes = 0;
        for (int i = 0; i < count; i++) limb_bytes += 8.0 * (double)(jobs.j[i].na + (square ? 0 : jobs.j[i].nb));
        e = launch_four_step(g.P3, G, jobs, (uint32_t)count, st, limb_bytes);
        if (e) return fail(FFG_E_CUDA, "four_step: %s", cudaGetErrorString(e));
    }
    CrtJob crt[FFG_FS_JOBS];
    for (int i = 0; i < count; i++) {
        CrtJob &C = crt[i];
        C = CrtJob{};
        C.y = ya[i];
        C.y_stride = L;
        uint64_t ca = (pr[i].bits_a + w - 1) / w, cb = square ? ca : (pr[i].bits_b + w - 1) / w;
        C.conv = ca + cb - 1;
        C.out = pr[i].out;
        C.nlimbs = pr[i].na + (square ? pr[i].na : pr[i].nb) + 1;
        C.width = w;
        C.add = pr[i].add;
        C.maps = (uint32_t *)arena_alloc((size_t)crt_ctas(C.nlimbs, w) * sizeof(uint32_t));
        if (!C.maps) return fail(FFG_E_NOMEM, "device arena: CRT scratch");
        C.ticket = ticket_get();
    }
    if (fuse && count == 2) {
        CrtLinJob F{};
        for (int q = 0; q < 2; q++) {
            F.y[q] = crt[q].y;
            F.conv[q] = crt[q].conv;
            F.out[q] = fuse->out[q];
            F.alpha[q] = fuse->alpha[q];
            F.beta[q] = fuse->beta[q];
            F.gamma[q] = fuse->gamma[q];
        }
        F.y_stride = L;
        F.len = fuse->len;
        F.width = w;
        F.maps = (uint32_t *)arena_alloc(2 * (size_t)crt_ctas(F.len, w) * sizeof(uint32_t));
        if (!F.maps) return fail(FFG_E_NOMEM, "device arena: CRT scratch");
        F.ticket = ticket_get();
        e = launch_crt_lin(F, st);
        if (e) return fail(FFG_E_CUDA, "crt + linear pass: %s", cudaGetErrorString(e));
        return FFG_OK;
    }
    for (int i = 0; i < count; i += 2) { // the step's pair in one launch
        e = launch_crt_pair(crt + i, count - i >= 2 ? 2 : 1, st);
        if (e) return fail(FFG_E_CUDA, "crt: %s", cudaGetErrorString(e));
    }
    return FFG_OK;
}

// The piecewise split multiply (src/mul_split.c:98-187) on the device: every
// piece of H = Lp/2 coefficients transformed once; per output piece m the
// pointwise sum over i + j = m, one inverse, added into the product's
// residues at m H; then one CRT over all of them.
int run_split(const Prod &pr, bool square, const ffg_plan &pl, cudaStream_t st) {
    const uint64_t Lp = pl.L, H = Lp / 2, ka = pl.ka, kb = pl.kb, Lyst = pl.Lbig + Lp;
    const uint32_t w = pl.width;
    FourStep G = four_step_geometry(pl, true);
    ALLOC(A, uint32_t, ka * 3 * Lp);
    uint32_t *B = A;
    if (!square) {
        ALLOC(Bt, uint32_t, kb * 3 * Lp);
        B = Bt;
    }
    ALLOC(Cb, uint32_t, 3 * Lp);
    ALLOC(Y, uint32_t, 3 * Lyst);
    CK(cudaMemsetAsync(Y, 0, 3 * Lyst * sizeof(uint32_t), st));
    const uint64_t np = ka + (square ? 0 : kb), nm = ka + kb - 1;
    std::vector<FSJob> jobs(np + nm);
    double limb_bytes = 0;
    for (uint64_t i = 0; i < np; i++) {
        const bool isb = i >= ka;
        const uint64_t k = isb ? i - ka : i, tot = isb ? pl.cb : pl.ca;
        FSJob &J = jobs[i];
        J.a = isb ? pr.b : pr.a;
        J.na = isb ? pr.nb : pr.na;
        J.off_a = k * H;
        J.ca = tot > k * H ? std::min(H, tot - k * H) : 0;
        J.ya = (isb ? B : A) + k * 3 * Lp;
        J.width = w;
        limb_bytes += (double)J.ca * w / 8.0;
    }
    for (uint64_t m = 0; m < nm; m++) {
        FSJob &J = jobs[np + m];
        J.pa = A;
        J.pb = B;
        J.piece_stride = 3 * Lp;
        J.m = (uint32_t)m, J.ka = (uint32_t)ka, J.kb = (uint32_t)kb, J.psq = square;
        J.ya = Cb;
        J.yacc = Y;
        J.acc_off = m * H;
        J.acc_stride = Lyst;
        J.width = w;
    }
    cudaError_t e = cudaSuccess;
    for (uint64_t f = 0; f < np; f += FFG_FS_JOBS) {
        FSJobs part{};
        const uint64_t cnt = std::min<uint64_t>(FFG_FS_JOBS, np - f);
        double lb = 0;
        for (uint64_t k = 0; k < cnt; k++) {
            part.j[k] = jobs[f + k];
            lb += (double)jobs[f + k].ca * w / 8.0;
        }
        e = launch_split_forward(g.P3, G, part, (uint32_t)cnt, st, lb);
        if (e) return fail(FFG_E_CUDA, "split forward: %s", cudaGetErrorString(e));
    }
    (void)limb_bytes;
    for (uint64_t m = 0; m < nm; m++) {
        const uint64_t i0 = m + 1 > kb ? m + 1 - kb : 0, i1 = std::min(m, ka - 1);
        e = launch_split_piece(g.P3, G, jobs[np + m], (uint32_t)(i1 - i0 + 1), st);
        if (e) return fail(FFG_E_CUDA, "split piece %llu: %s", (unsigned long long)m, cudaGetErrorString(e));
    }
    CrtJob C{};
    C.y = Y;
    C.y_stride = Lyst;
    C.conv = pl.conv;
    C.out = pr.out;
    C.nlimbs = pr.na + (square ? pr.na : pr.nb) + 1;
    C.width = w;
    C.add = pr.add;
    C.maps = (uint32_t *)arena_alloc((size_t)crt_ctas(C.nlimbs, w) * sizeof(uint32_t));
    if (!C.maps) return fail(FFG_E_NOMEM, "device arena: CRT scratch");
    C.ticket = ticket_get();
    e = launch_crt(g.P3, C, st);
    if (e) return fail(FFG_E_CUDA, "crt: %s", cudaGetErrorString(e));
    return FFG_OK;
}

// One product on device limbs (plan from the bit lengths).
static int mul_one(const Prod &p, bool square, cudaStream_t st) {
    ffg_plan pl;
    int rc = plan_select(p.bits_a, square ? p.bits_a : p.bits_b, square, &pl);
    if (rc) return rc;
    if (pl.split) return run_split(p, square, pl, st);
    return run_products(&p, 1, pl, square, st);
}

uint64_t bits_of(const uint64_t *a, size_t n) {
    while (n > 0 && a[n - 1] == 0) n--;
    if (n == 0) return 0;
    return 64 * (n - 1) + (64 - (uint64_t)__builtin_clzll(a[n - 1]));
}

// -------------------------------------------------------- fast doubling

static const long double kLog2Phi = 0.6942419136306174017387902668985552L;
static const long double kLog2Sqrt5 = 1.1609640474436811739351597147446950L;

// Bit length of F(m) (m >= 2): floor(m log2(phi) - log2(sqrt 5)) + 1, since
// F(m) = round(phi^m / sqrt 5).  When the value sits too close to an integer
// for long double to decide, one more bit is returned (a safe upper bound).
static uint64_t fib_bits(uint64_t m) {
    long double x = (long double)m * kLog2Phi - kLog2Sqrt5, f = floorl(x);
    uint64_t b = (uint64_t)f + 1;
    if (x - f < 1e-7L || f + 1 - x < 1e-7L) b++;
    return b;
}
// Bit length of the Lucas number L(m) = round(phi^m) (m >= 2), same guard.
static uint64_t lucas_bits(uint64_t m) {
    long double x = (long double)m * kLog2Phi, f = floorl(x);
    uint64_t b = (uint64_t)f + 1;
    if (x - f < 1e-7L || f + 1 - x < 1e-7L) b++;
    return b;
}

static int lin(const uint64_t *s1, uint64_t n1, const uint64_t *s2, uint64_t n2, uint64_t len, int nout,
               uint64_t *o0, int a0, int b0, int64_t g0, uint64_t *o1, int a1, int b1, int64_t g1, cudaStream_t st) {
    LinJob J{};
    J.s1 = s1, J.s2 = s2, J.n1 = n1, J.n2 = n2, J.len = len;
    J.out[0] = o0, J.out[1] = o1;
    J.alpha[0] = a0, J.beta[0] = b0, J.gamma[0] = g0;
    J.alpha[1] = a1, J.beta[1] = b1, J.gamma[1] = g1;
    J.nout = (uint32_t)nout;
    J.maps = (uint32_t *)arena_alloc(2 * (size_t)lin_ctas(len) * sizeof(uint32_t));
    J.ticket = ticket_get();
    if (!J.maps) return fail(FFG_E_NOMEM, "device arena: linear pass scratch");
    cudaError_t e = launch_lin(J, st);
    if (e) return fail(FFG_E_CUDA, "linear pass: %s", cudaGetErrorString(e));
    return FFG_OK;
}

// FFG_NO_CRT_LIN=1: the step's CRT pair and linear pass as two launches
// (the same results; for comparing the two).
static bool crt_lin_enabled() {
    static int on = -1;
    if (on < 0) {
        const char *e = getenv("FFG_NO_CRT_LIN");
        on = !(e && *e && *e != '0');
    }
    return on != 0;
}

// The device part of the chain, from the pair (F(k-1), F(k)) in fkm1 / fk
// (bit lengths bkm1 / bk) to F(n) in *res (*nres limbs, leading zeros
// allowed): kernel launches and arena allocations only, in the same order on
// every call, so a CUDA graph can capture it.
static int chain_body(uint64_t n, int i0, uint64_t *fk, uint64_t *fkm1, uint64_t bk, uint64_t bkm1,
                      uint64_t **res_out, uint64_t *nres_out, cudaStream_t st) {
    uint64_t k = n >> i0;
    int kodd = (int)(k & 1);
    uint64_t nk, nkm1;
    for (int i = i0 - 1; i >= 1; i--) {
        const int bit = (int)((n >> i) & 1);
        if (bkm1 == 0) bkm1 = 1;
        nk = (bk + 63) / 64, nkm1 = (bkm1 + 63) / 64;
        const uint64_t n1 = 2 * nk + 1, n2 = 2 * nkm1 + 1;
        ALLOC(s1, uint64_t, n1);
        ALLOC(s2, uint64_t, n2);
        Prod p1{fk, fk, nk, nk, bk, bk, s1, 0}, p2{fkm1, fkm1, nkm1, nkm1, bkm1, bkm1, s2, 0};
        ffg_plan pl1, pl2;
        int rc = plan_select(bk, bk, 1, &pl1);
        if (!rc) rc = plan_select(bkm1, bkm1, 1, &pl2);
        if (rc) return rc;
        if (nk <= kChainSchoolLimbs) {
            // short operands: both squarings as schoolbook products, one launch
            SchoolJob sj[2];
            const Prod *pp[2] = {&p1, &p2};
            for (int q = 0; q < 2; q++) {
                SchoolJob &J = sj[q];
                J = SchoolJob{};
                J.a = J.b = pp[q]->a;
                J.na = J.nb = (pp[q]->bits_a + 63) / 64;
                J.out = pp[q]->out;
                J.nlimbs = 2 * pp[q]->na + 1;
                J.maps = (uint32_t *)arena_alloc((size_t)school_sq_ctas(J.nlimbs) * 4);
                if (!J.maps) return fail(FFG_E_NOMEM, "device arena: schoolbook maps");
                J.ticket = ticket_get();
            }
            cudaError_t e = launch_school_sq_pair(sj, 2, st);
            if (e) return fail(FFG_E_CUDA, "schoolbook pair: %s", cudaGetErrorString(e));
        } else if (pl1.split || pl2.split) {
            rc = mul_one(p1, true, st);
            if (!rc) rc = mul_one(p2, true, st);
        } else if (pl1.width == pl2.width && pl1.L == pl2.L && pl1.kernel == pl2.kernel &&
                   pl1.row_lg == pl2.row_lg && crt_lin_enabled()) {
            // both squarings in one launch set; the CRT writes the step's
            // two results directly (k_crt_lin)
            Prod pp[2] = {p1, p2};
            const uint64_t len = n1 + 1;
            const int64_t pm2 = kodd ? -2 : 2;
            ALLOC(lo, uint64_t, len);
            ALLOC(hi, uint64_t, len);
            LinFuse fz{};
            fz.out[0] = lo, fz.out[1] = hi, fz.len = len;
            if (bit) {
                fz.alpha[0] = 3, fz.beta[0] = -2, fz.gamma[0] = pm2;
                fz.alpha[1] = 4, fz.beta[1] = -1, fz.gamma[1] = pm2;
            } else {
                fz.alpha[0] = 1, fz.beta[0] = 1, fz.gamma[0] = 0;
                fz.alpha[1] = 3, fz.beta[1] = -2, fz.gamma[1] = pm2;
            }
            rc = run_products(pp, 2, pl1, true, st, &fz);
            if (rc) return rc;
            k = 2 * k + (uint64_t)bit;
            kodd = bit;
            fkm1 = lo;
            fk = hi;
            bk = fib_bits(k);
            bkm1 = fib_bits(k - 1);
            continue;
        } else if (pl1.width == pl2.width && pl1.L == pl2.L && pl1.kernel == pl2.kernel &&
                   pl1.row_lg == pl2.row_lg) {
            Prod pp[2] = {p1, p2};
            rc = run_products(pp, 2, pl1, true, st);
        } else {
            rc = run_products(&p1, 1, pl1, true, st);
            if (!rc) rc = run_products(&p2, 1, pl2, true, st);
        }
        if (rc) return rc;
        // A = s1 + s2 = F(2k-1), B = 4 s1 - s2 + 2(-1)^k = F(2k+1), C = B - A = F(2k)
        const uint64_t len = n1 + 1;
        const int64_t pm2 = kodd ? -2 : 2;
        ALLOC(lo, uint64_t, len);
        ALLOC(hi, uint64_t, len);
        if (bit) rc = lin(s1, n1, s2, n2, len, 2, lo, 3, -2, pm2, hi, 4, -1, pm2, st);
        else rc = lin(s1, n1, s2, n2, len, 2, lo, 1, 1, 0, hi, 3, -2, pm2, st);
        if (rc) return rc;
        k = 2 * k + (uint64_t)bit;
        kodd = bit;
        fkm1 = lo;
        fk = hi;
        bk = fib_bits(k);
        bkm1 = fib_bits(k - 1);
    }
    // last bit (src/fib.c:239-260)
    nk = (bk + 63) / 64, nkm1 = (bkm1 + 63) / 64;
    const uint64_t lenx = std::max(nk, nkm1) + 1;
    uint64_t *res = nullptr;
    uint64_t nres = 0;
    int rc;
    if (n & 1) {
        ALLOC(x, uint64_t, lenx);
        ALLOC(y, uint64_t, lenx);
        rc = lin(fk, nk, fkm1, nkm1, lenx, 2, x, 2, 1, 0, y, 2, -1, 0, st);
        if (rc) return rc;
        uint64_t bx = fib_bits(k + 2);   // 2F(k) + F(k-1) = F(k+2)
        uint64_t by = lucas_bits(k - 1); // 2F(k) - F(k-1) = F(k) + F(k-2) = L(k-1)
        nres = 2 * lenx + 1;
        ALLOC(r, uint64_t, nres);
        res = r;
        Prod p{x, y, lenx, lenx, bx, by, r, kodd ? -2 : 2};
        rc = mul_one(p, false, st);
    } else {
        ALLOC(x, uint64_t, lenx);
        rc = lin(fkm1, nkm1, fk, nk, lenx, 1, x, 2, 1, 0, nullptr, 0, 0, 0, st);
        if (rc) return rc;
        uint64_t bx = lucas_bits(k); // F(k) + 2F(k-1) = L(k)
        nres = nk + lenx + 1;
        ALLOC(r, uint64_t, nres);
        res = r;
        Prod p{fk, x, nk, lenx, bk, bx, r, 0};
        rc = mul_one(p, false, st);
    }
    if (rc) return rc;
    *res_out = res;
    *nres_out = nres;
    return FFG_OK;
}

// A captured chain for one n (and one starting pair size), replayed by later
// calls: the pair is copied into the same device buffers and the graph runs.
struct ChainGraph {
    uint64_t n;
    int i0;
    uint64_t max_L;   // plans depend on the transform cap
    uint64_t hnk, hnkm1;
    uint32_t prof_mask;
    uint64_t *fk, *fkm1, *res;
    uint64_t nres;
    int eager_runs;
    cudaGraphExec_t exec;
    uint64_t launches;
    std::vector<ProfPair> prof;
};
static std::vector<ChainGraph> g_chains;

void chain_cache_clear() {
    for (auto &c : g_chains)
        if (c.exec) cudaGraphExecDestroy(c.exec);
    g_chains.clear();
}

// Results come back to the host in pinned buffers (a DMA straight into the
// caller's memory, no staging copy).  They are pooled: ffg_free / ffg_release
// return one to the pool, and the next result of a fitting size reuses it.
static std::vector<std::pair<void *, size_t>> g_pinned_out, g_pinned_pool;
static volatile size_t g_pinned_outstanding = 0;

void *pinned_get(size_t bytes) {
    size_t best = (size_t)-1;
    for (size_t i = 0; i < g_pinned_pool.size(); i++)
        if (g_pinned_pool[i].second >= bytes &&
            (best == (size_t)-1 || g_pinned_pool[i].second < g_pinned_pool[best].second))
            best = i;
    std::pair<void *, size_t> b;
    if (best != (size_t)-1) {
        b = g_pinned_pool[best];
        g_pinned_pool.erase(g_pinned_pool.begin() + best);
    } else {
        size_t cap = std::max(bytes, (size_t)1 << 20);
        void *p = nullptr;
        if (cudaMallocHost(&p, cap) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        b = {p, cap};
    }
    g_pinned_out.push_back(b);
    g_pinned_outstanding = g_pinned_out.size();
    return b.first;
}

// Returns 1 if p is a pooled result buffer (now back in the pool), else 0.
int pinned_release(void *p) {
    for (size_t i = 0; i < g_pinned_out.size(); i++)
        if (g_pinned_out[i].first == p) {
            g_pinned_pool.push_back(g_pinned_out[i]);
            g_pinned_out.erase(g_pinned_out.begin() + i);
            g_pinned_outstanding = g_pinned_out.size();
            return 1;
        }
    return 0;
}

static bool graphs_enabled() {
    const char *e = getenv("FFG_NO_GRAPH");
    return !(e && *e && *e != '0');
}

static int fib_chain(uint64_t n, int i0, const uint64_t *hkm1, size_t hnkm1, const uint64_t *hk, size_t hnk,
                     uint64_t **out, size_t *nout) {
    cudaStream_t st = g.stream;
    const uint64_t nk = hnk ? hnk : 1, nkm1 = hnkm1 ? hnkm1 : 1;
    const uint64_t cap0 = std::max(nk, nkm1);
    ALLOC(fk, uint64_t, cap0);
    ALLOC(fkm1, uint64_t, cap0);
    CK(cudaMemsetAsync(fk, 0, cap0 * 8, st));
    CK(cudaMemsetAsync(fkm1, 0, cap0 * 8, st));
    CK(cudaMemcpyAsync(fk, hk, hnk * 8, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(fkm1, hkm1, hnkm1 * 8, cudaMemcpyHostToDevice, st));
    const uint64_t bk = bits_of(hk, hnk), bkm1 = bits_of(hkm1, hnkm1);
    const uint32_t mask = g_prof_on ? g_prof_mask : 0;

    ChainGraph *cg = nullptr;
    for (auto &c : g_chains)
        if (c.n == n && c.i0 == i0 && c.max_L == g.max_L && c.hnk == hnk && c.hnkm1 == hnkm1 &&
            c.prof_mask == mask)
            cg = &c;
    uint64_t *res = nullptr, nres = 0;
    if (cg && cg->exec && cg->fk == fk && cg->fkm1 == fkm1) {
        CK(cudaEventRecord(g.ev0, st));
        CK(cudaGraphLaunch(cg->exec, st));
        CK(cudaEventRecord(g.ev1, st));
        g_launches += cg->launches;
        res = cg->res;
        nres = cg->nres;
    } else {
        bool capture = graphs_enabled() && cg && cg->eager_runs >= 1 && cg->fk == fk && cg->fkm1 == fkm1;
        const uint64_t launches0 = g_launches;
        const size_t prof0 = g_prof_open.size();
        const auto marks = g.blocks; // arena state after the pair, to rerun eagerly from
        CK(cudaEventRecord(g.ev0, st));
        int rc = FFG_OK;
        if (capture) {
            CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            g_capturing = true;
            rc = chain_body(n, i0, fk, fkm1, bk, bkm1, &res, &nres, st);
            g_capturing = false;
            cudaGraph_t graph = nullptr;
            cudaError_t e = cudaStreamEndCapture(st, &graph);
            cudaGraphExec_t exec = nullptr;
            if (!rc && e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
            if (graph) cudaGraphDestroy(graph);
            if (rc || e != cudaSuccess) {
                // abandoned (e.g. the arena would have had to grow): run eagerly
                cudaGetLastError();
                if (exec) cudaGraphExecDestroy(exec);
                for (size_t b = 0; b < g.blocks.size(); b++) g.blocks[b].used = b < marks.size() ? marks[b].used : 0;
                for (size_t q = prof0; q < g_prof_open.size(); q++) {
                    g_ev_pool.push_back(g_prof_open[q].a);
                    if (g_prof_open[q].b) g_ev_pool.push_back(g_prof_open[q].b);
                }
                g_prof_open.resize(prof0);
                g_launches = launches0;
                capture = false;
            }
            if (!capture) {
                rc = chain_body(n, i0, fk, fkm1, bk, bkm1, &res, &nres, st);
                if (rc) return rc;
                cg->eager_runs++;
                CK(cudaEventRecord(g.ev1, st));
                goto copy_back;
            }
            cg->exec = exec;
            cg->res = res;
            cg->nres = nres;
            cg->launches = g_launches - launches0;
            // the captured event brackets belong to the graph from now on
            cg->prof.assign(g_prof_open.begin() + prof0, g_prof_open.end());
            g_prof_open.resize(prof0);
            CK(cudaGraphLaunch(exec, st));
        } else {
            rc = chain_body(n, i0, fk, fkm1, bk, bkm1, &res, &nres, st);
            if (rc) return rc;
            if (!cg) {
                if (g_chains.size() >= 8) {
                    if (g_chains.front().exec) cudaGraphExecDestroy(g_chains.front().exec);
                    g_chains.erase(g_chains.begin());
                }
                g_chains.push_back(ChainGraph{n, i0, g.max_L, hnk, hnkm1, mask, fk, fkm1, nullptr, 0, 0, nullptr, 0, {}});
                cg = &g_chains.back();
            }
            cg->eager_runs++;
        }
        CK(cudaEventRecord(g.ev1, st));
    }
copy_back:
    uint64_t *h = (uint64_t *)pinned_get(nres * 8);
    if (!h) return fail(FFG_E_NOMEM, "pinned host buffer: %zu bytes", (size_t)nres * 8);
    CK(cudaMemcpyAsync(h, res, nres * 8, cudaMemcpyDeviceToHost, st));
    cudaError_t e = cudaStreamSynchronize(st);
    if (e) {
        pinned_release(h);
        return fail(FFG_E_CUDA, "fib chain: %s", cudaGetErrorString(e));
    }
    if (cg && cg->exec) { // a replay (or the capture's first run): its brackets
        for (auto &pp : cg->prof) {
            float ms = 0;
            if (pp.b && cudaEventElapsedTime(&ms, pp.a, pp.b) == cudaSuccess) {
                g_prof_ms[pp.kind] += ms;
                g_prof_bytes[pp.kind] += pp.bytes;
                g_prof_n[pp.kind]++;
            }
        }
    }
    float ms = 0;
    cudaEventElapsedTime(&ms, g.ev0, g.ev1);
    g.chain_ms = ms;
    g.chain_h2d = 8 * (uint64_t)(hnk + hnkm1);
    g.chain_d2h = 8 * nres;
    while (nres > 1 && h[nres - 1] == 0) nres--;
    *out = h;
    *nout = nres;
    return FFG_OK;
}

} // namespace ffg

// =================================================================== C ABI

using namespace ffg;

static int noalloc_address(int dev, void **addr);

extern "C" int ffg_init(size_t max_limbs) {
    std::lock_guard<std::recursive_mutex> lk(g_mu);
    int rc = ensure_ready();
    if (rc) return rc;
    // the allocation-free multiply's scratch address, looked up now: the
    // lookup loads the module holding the array (which places it on the
    // device), so that entry point allocates nothing even on its first call
    int dev = 0;
    CK(cudaGetDevice(&dev));
    void *scratch = nullptr;
    if ((rc = noalloc_address(dev, &scratch))) return rc;
    CK(ntt_kernels_load()); // and the kernels it launches, for the same reason
    CK(crt_kernel_load());
    size_t L = 16;
    while (L < 2 * max_limbs && L < ((size_t)1 << kMaxLg)) L <<= 1;
    if (L > g.max_L) g.max_L = L;
    return FFG_OK;
}

extern "C" size_t ffg_ntt_max_L(void) { return g.max_L; }

extern "C" int ffg_set_max_lg(int lg) {
    std::lock_guard<std::recursive_mutex> lk(g_mu);
    if (lg < 4 || lg > 25) return fail(FFG_E_ARG, "max lg %d outside 4..25", lg);
    kMaxLg = lg;
    if (g.max_L > ((size_t)1 << lg)) g.max_L = (size_t)1 << lg;
    return FFG_OK;
}
extern "C" void ffg_set_ntt_max_L(size_t L) { g.max_L = L; }

extern "C" int ffg_plan_select(uint64_t bits_a, uint64_t bits_b, int square, ffg_plan *plan) {
    std::lock_guard<std::recursive_mutex> lk(g_mu);
    if (!plan) return fail(FFG_E_ARG, "plan is NULL");
    int rc = plan_select(bits_a, bits_b, square, plan);
    return rc;
}

extern "C" int ffg_mul_device(uint64_t *out, const uint64_t *a, size_t na, uint64_t bits_a, const uint64_t *b,
                              size_t nb, uint64_t bits_b, int square, void *stream) {
    std::lock_guard<std::recursive_mutex> lk(g_mu);
    int rc = ensure_ready();
    if (rc) return rc;
    if (!out || !a || (!square && !b) || na == 0 || (!square && nb == 0)) return fail(FFG_E_ARG, "bad arguments");
    cudaStream_t st = stream ? (cudaStream_t)stream : g.stream;
    Prod p{a, square ? a : b, na, square ? na : nb, bits_a, square ? bits_a : bits_b, out, 0};
    if (bits_a == 0 || (!square && bits_b == 0)) {
        CK(cudaMemsetAsync(out, 0, (na + (square ? na : nb) + 1) * 8, st));
        return FFG_OK;
    }
    arena_reset();
    return mul_one(p, square != 0, st);
}

extern "C" int ffg_mul_host(uint64_t *out, size_t *nout, const uint64_t *a, size_t na, const uint64_t *b, size_t nb,
                            int square) {
    std::lock_guard<std::recursive_mutex> lk(g_mu);
    int rc = ensure_ready();
    if (rc) return rc;
    if (square) b = a, nb = na;
    uint64_t ba = bits_of(a, na), bb = bits_of(b, nb);
    if (ba == 0 || bb == 0) {
        out[0] = 0;
        *nout = 1;
        return FFG_OK;
    }
    na = (ba + 63) / 64, nb = (bb + 63) / 64;
    cudaStream_t st = g.stream;
    CK(cudaStreamSynchronize(st));
    arena_reset();
    ALLOC(da, uint64_t, na);
    uint64_t *db = da;
    if (!square) {
        ALLOC(t, uint64_t, nb);
        db = t;
    }
    const uint64_t nr = na + nb + 1;
    ALLOC(dr, uint64_t, nr);
    CK(cudaMemcpyAsync(da, a, na * 8, cudaMemcpyHostToDevice, st));
    if (!square) CK(cudaMemcpyAsync(db, b, nb * 8, cudaMemcpyHostToDevice, st));
    Prod p{da, db, na, nb, ba, bb, dr, 0};
    rc = mul_one(p, square != 0, st);
    if (rc) return rc;
    std::vector<uint64_t> tmp(nr);
    CK(cudaMemcpyAsync(tmp.data(), dr, nr * 8, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    size_t n = na + nb;
    while (n > 1 && tmp[n - 1] == 0) n--;
    memcpy(out, tmp.data(), n * 8);
    *nout = n;
    return FFG_OK;
}

extern "C" int ffg_fib_chain(uint64_t n, int i0, const uint64_t *fkm1, size_t nkm1, const uint64_t *fk, size_t nk,
                             uint64_t **out, size_t *nout) {
    std::lock_guard<std::recursive_mutex> lk(g_mu);
    int rc = ensure_ready();
    if (rc) return rc;
    if (i0 < 1 || i0 > 63 || !fk || !out || !nout) return fail(FFG_E_ARG, "bad arguments");
    CK(cudaStreamSynchronize(g.stream));
    arena_reset();
    return fib_chain(n, i0, fkm1, nkm1, fk, nk, out, nout);
}

extern "C" double ffg_last_chain_ms(void) { return g.chain_ms; }

extern "C" void ffg_last_chain_io(uint64_t *h2d_bytes, uint64_t *d2h_bytes) {
    *h2d_bytes = g.chain_h2d;
    *d2h_bytes = g.chain_d2h;
}

extern "C" int ffg_set_device(int device) {
    std::lock_guard<std::recursive_mutex> lk(g_mu);
    if (g.ready && device != g.device) return fail(FFG_E_ARG, "device already chosen (%d)", g.device);
    g.device = device;
    if (!g.ready) return FFG_OK;
    CK(cudaSetDevice(device));
    return FFG_OK;
}

extern "C" void ffg_profile(uint32_t mask) {
    std::lock_guard<std::recursive_mutex> lk(g_mu);
    prof_collect();
    g_prof_on = mask != 0;
    g_prof_mask = mask;
    for (int k = 0; k < PK_COUNT; k++) g_prof_ms[k] = g_prof_bytes[k] = 0, g_prof_n[k] = 0;
}

extern "C" int ffg_profile_read(int kind, uint64_t *launches, double *ms, double *bytes) {
    std::lock_guard<std::recursive_mutex> lk(g_mu);
    if (kind < 0 || kind >= PK_COUNT) return fail(FFG_E_ARG, "profile kind %d", kind);
    prof_collect();
    *launches = g_prof_n[kind];
    *ms = g_prof_ms[kind];
    *bytes = g_prof_bytes[kind];
    return FFG_OK;
}

extern "C" uint64_t ffg_launch_count(void) { return g_launches; }
extern "C" const char *ffg_last_error(void) { return g.err.c_str(); }
extern "C" int ffg_release(void *p) {
    if (!p || !g_pinned_outstanding) return 0;
    std::lock_guard<std::recursive_mutex> lk(g_mu);
    return pinned_release(p);
}

extern "C" void ffg_free(void *p) {
    if (!ffg_release(p)) free(p);
}

static void *g_noalloc_addr[64]; // the allocation-free scratch's device address, per device

extern "C" void ffg_shutdown(void) {
    std::lock_guard<std::recursive_mutex> lk(g_mu);
    if (!g.ready) return;
    cudaStreamSynchronize(g.stream);
    chain_cache_clear();
    for (auto &b : g.blocks) cudaFree(b.ptr);
    g.blocks.clear();
    cudaFree(g.tables);
    g.tables = nullptr;
    mlp_free();
    lanes_free();
    if (g_tickets) cudaFree(g_tickets);
    g_tickets = nullptr;
    dec_free();
    for (auto &b : g_pinned_pool) cudaFreeHost(b.first);
    g_pinned_pool.clear();
    cudaEventDestroy(g.ev0);
    cudaEventDestroy(g.ev1);
    cudaStreamDestroy(g.stream);
    g.ready = false;
    for (auto &a : g_noalloc_addr) a = nullptr; // looked up again by the next ffg_init
}

// ======================================================= prime sharding
//
// One product over several GPUs by prime: a rank transforms, multiplies and
// inverts its primes only (the four-step launches over a range of primes,
// FourStep::prime0 / nprimes), the ranks exchange their slices of the
// residues (the caller's all-gather, 4 L bytes a prime), and the CRT runs on
// the gathered array.  The primes' transforms are independent, so that
// all-gather is the one exchange.

// The product's plan, when it is one prime sharding takes (a four-step plan).
static int residue_plan(uint64_t bits_a, uint64_t bits_b, int square, ffg_plan *pl) {
    int rc = plan_select(bits_a, bits_b, square, pl);
    if (rc) return rc;
    if (pl->split) return fail(FFG_E_RANGE, "prime sharding: a split product (past the transform cap)");
    if (pl->kernel == 0)
        return fail(FFG_E_RANGE, "prime sharding: length %llu is a one-CTA transform (four-step lengths only)",
                    (unsigned long long)pl->L);
    return FFG_OK;
}

extern "C" int ffg_mul_residues(uint32_t *y, const uint64_t *a, size_t na, uint64_t bits_a, const uint64_t *b,
                                size_t nb, uint64_t bits_b, int square, uint32_t prime0, uint32_t nprimes,
                                void *stream) {
    std::lock_guard<std::recursive_mutex> lk(g_mu);
    int rc = ensure_ready();
    if (rc) return rc;
    if (!y || !a || (!square && !b) || na == 0 || (!square && nb == 0) || bits_a == 0 || (!square && bits_b == 0))
        return fail(FFG_E_ARG, "ffg_mul_residues: bad arguments");
    if (nprimes == 0 || prime0 >= 3 || nprimes > 3 - prime0)
        return fail(FFG_E_ARG, "ffg_mul_residues: primes [%u, %u + %u) outside [0, 3)", prime0, prime0, nprimes);
    if (square) b = a, nb = na, bits_b = bits_a;
    ffg_plan pl;
    if ((rc = residue_plan(bits_a, bits_b, square, &pl))) return rc;
    cudaStream_t st = stream ? (cudaStream_t)stream : g.stream;
    arena_reset();
    const uint64_t L = pl.L;
    const uint32_t w = pl.width;
    FourStep G = four_step_geometry(pl, square != 0);
    G.prime0 = prime0;
    G.nprimes = nprimes;
    FSJobs jobs{};
    FSJob &J = jobs.j[0];
    J.a = a, J.b = b, J.na = na, J.nb = nb;
    J.ca = (bits_a + w - 1) / w;
    J.cb = (bits_b + w - 1) / w;
    J.ya = y;
    J.yb = square ? nullptr : (uint32_t *)arena_alloc(3 * L * sizeof(uint32_t));
    if (!square && !J.yb) return fail(FFG_E_NOMEM, "device arena: residues of L=%llu", (unsigned long long)L);
    J.width = w;
    cudaError_t e = launch_four_step(g.P3, G, jobs, 1, st, 8.0 * (double)(na + (square ? 0 : nb)));
    if (e) return fail(FFG_E_CUDA, "ffg_mul_residues: %s", cudaGetErrorString(e));
    return FFG_OK;
}

extern "C" int ffg_crt_residues(uint64_t *out, const uint32_t *y, size_t na, uint64_t bits_a, size_t nb,
                                uint64_t bits_b, int square, void *stream) {
    std::lock_guard<std::recursive_mutex> lk(g_mu);
    int rc = ensure_ready();
    if (rc) return rc;
    if (!out || !y || na == 0 || (!square && nb == 0) || bits_a == 0 || (!square && bits_b == 0))
        return fail(FFG_E_ARG, "ffg_crt_residues: bad arguments");
    if (square) nb = na, bits_b = bits_a;
    ffg_plan pl;
    if ((rc = residue_plan(bits_a, bits_b, square, &pl))) return rc;
    cudaStream_t st = stream ? (cudaStream_t)stream : g.stream;
    arena_reset();
    const uint32_t w = pl.width;
    CrtJob C{};
    C.y = y;
    C.y_stride = pl.L;
    C.conv = (bits_a + w - 1) / w + (bits_b + w - 1) / w - 1;
    C.out = out;
    C.nlimbs = na + nb + 1;
    C.width = w;
    C.add = 0;
    C.maps = (uint32_t *)arena_alloc((size_t)crt_ctas(C.nlimbs, w) * sizeof(uint32_t));
    if (!C.maps) return fail(FFG_E_NOMEM, "device arena: CRT scratch");
    C.ticket = ticket_get();
    cudaError_t e = launch_crt(g.P3, C, st);
    if (e) return fail(FFG_E_CUDA, "ffg_crt_residues: %s", cudaGetErrorString(e));
    return FFG_OK;
}

// ======================================================= allocation-free multiply
//
// ffg_mul_device_noalloc: the NTT product of ffg_mul_device for callers that
// must not allocate device memory once they are running -- a host program
// whose device memory is all owned by another allocator (a framework's
// caching allocator, a fixed budget handed out at start-up), or a
// latency-critical path that cannot afford a cudaMalloc (and the device-wide
// synchronization it may imply).  Its scratch (the residue arrays, the job record and the CRT's carry
// maps) lives in the fixed array below, which every GPU that loads this
// library holds until the process exits; products whose scratch would not fit
// are rejected with FFG_E_RANGE.  The device tables are built once by
// ffg_init, which the caller runs during its own set-up and which also looks
// up the array's device address and loads the kernels used here; this entry
// point itself calls no cudaMalloc, cudaFree or other allocating routine.

static constexpr size_t kNoAllocBytes = (size_t)8 << 20; // 8 MiB per device
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];
// Host code may not use g_noalloc_scratch's name as an address (it is a host
// stand-in); the device address comes from cudaGetSymbolAddress, looked up
// once per device with that device current.
static int noalloc_address(int dev, void **addr) {
    if (dev < 0 || dev >= 64) return fail(FFG_E_ARG, "device %d out of range", dev);
    if (!g_noalloc_addr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess)
            return fail(FFG_E_CUDA, "cudaGetSymbolAddress(allocation-free scratch): %s", cudaGetErrorString(e));
        g_noalloc_addr[dev] = p;
    }
    *addr = g_noalloc_addr[dev];
    return FFG_OK;
}

static size_t up256(size_t x) { return (x + 255) & ~(size_t)255; }

extern "C" int ffg_mul_device_noalloc(uint64_t *out, const uint64_t *a, size_t na, uint64_t bits_a,
                                      const uint64_t *b, size_t nb, uint64_t bits_b, int square, void *stream) {
    std::lock_guard<std::recursive_mutex> lk(g_mu);
    if (!g.ready) return fail(FFG_E_ARG, "ffg_mul_device_noalloc: call ffg_init during set-up first");
    if (!out || !a || (!square && !b) || na == 0 || (!square && nb == 0)) return fail(FFG_E_ARG, "bad arguments");
    if (g.device >= 0) CK(cudaSetDevice(g.device));
    int dev = 0;
    CK(cudaGetDevice(&dev));
    void *base = nullptr;
    int rc = noalloc_address(dev, &base);
    if (rc) return rc;
    cudaStream_t st = stream ? (cudaStream_t)stream : g.stream;
    if (square) b = a, nb = na, bits_b = bits_a;
    const uint64_t nlimbs = na + nb + 1;
    if (bits_a == 0 || bits_b == 0) {
        CK(cudaMemsetAsync(out, 0, nlimbs * 8, st));
        return FFG_OK;
    }
    ffg_plan pl;
    rc = plan_select(bits_a, bits_b, square, &pl);
    if (rc) return rc;
    if (pl.split) return fail(FFG_E_RANGE, "ffg_mul_device_noalloc: the product needs the split multiply");

    // scratch layout: residues of a | residues of b | CRT carry maps
    const uint64_t L = pl.L;
    const uint32_t w = pl.width;
    const size_t o_ya = 0;
    const size_t o_yb = o_ya + up256(3 * L * sizeof(uint32_t));
    const size_t o_maps = o_yb + (square ? 0 : up256(3 * L * sizeof(uint32_t)));
    const size_t need = o_maps + up256((size_t)crt_ctas(nlimbs, w) * sizeof(uint32_t));
    if (need > kNoAllocBytes)
        return fail(FFG_E_RANGE,
                    "ffg_mul_device_noalloc: %llu x %llu bits needs %zu bytes of scratch, the limit is %zu bytes",
                    (unsigned long long)bits_a, (unsigned long long)bits_b, need, kNoAllocBytes);
    char *s = (char *)base;
    uint32_t *ya = (uint32_t *)(s + o_ya), *yb = square ? nullptr : (uint32_t *)(s + o_yb);
    const uint64_t ca = (bits_a + w - 1) / w, cb = (bits_b + w - 1) / w;
    cudaError_t e;
    if (pl.kernel == 0) {
        ConvJobs jobs{};
        ConvJob &J = jobs.j[0];
        J.a = a, J.b = b, J.na = na, J.nb = nb, J.ca = ca, J.cb = cb;
        J.y = ya;
        J.y_stride = L;
        J.L_words = (uint32_t)L;
        J.n = pl.lg, J.r3 = pl.r3, J.width = w, J.square = square != 0;
        J.conv = (uint32_t)(ca + cb - 1);
        scale_consts(L, J.scl, J.scls);
        e = launch_conv_small(g.P3, jobs, 1, (uint32_t)L, !square, st,
                              8.0 * (double)(na + (square ? 0 : nb)) + 12.0 * (double)J.conv);
    } else {
        FourStep G = four_step_geometry(pl, square != 0);
        FSJobs jobs{};
        FSJob &J = jobs.j[0];
        J.a = a, J.b = b, J.na = na, J.nb = nb, J.ca = ca, J.cb = cb;
        J.ya = ya, J.yb = yb;
        J.width = w;
        e = launch_four_step(g.P3, G, jobs, 1, st, 8.0 * (double)(na + (square ? 0 : nb)));
    }
    if (e) return fail(FFG_E_CUDA, "ffg_mul_device_noalloc: %s", cudaGetErrorString(e));
    CrtJob C{};
    C.y = ya;
    C.y_stride = L;
    C.conv = ca + cb - 1;
    C.out = out;
    C.nlimbs = nlimbs;
    C.width = w;
    C.add = 0;
    C.maps = (uint32_t *)(s + o_maps);
    C.ticket = ticket_get_reserved();
    e = launch_crt(g.P3, C, st);
    if (e) return fail(FFG_E_CUDA, "ffg_mul_device_noalloc crt: %s", cudaGetErrorString(e));
    return FFG_OK;
}

// ------------------------------------------------------------ tuning

extern "C" int ffg_set_geometry(uint32_t lg, uint32_t r3, uint32_t row_lg, uint32_t wc) {
    std::lock_guard<std::recursive_mutex> lk(g_mu);
    if (lg >= 32 || r3 > 1) return fail(FFG_E_ARG, "geometry: lg %u r3 %u", lg, r3);
    if (row_lg == 0 && wc == 0) {
        g_geo[lg][r3] = Geo{0, 0, 0};
    } else {
        if (!geo_valid(lg, r3, row_lg, wc)) return fail(FFG_E_ARG, "geometry lg %u r3 %u: c %u wc %u", lg, r3, row_lg, wc);
        g_geo[lg][r3] = Geo{1, (uint8_t)row_lg, (uint8_t)wc};
    }
    chain_cache_clear(); // captured chains hold launches of the old geometry
    return FFG_OK;
}

extern "C" int ffg_get_geometry(uint32_t lg, uint32_t r3, uint32_t *row_lg, uint32_t *wc) {
    std::lock_guard<std::recursive_mutex> lk(g_mu);
    if (lg >= 32 || r3 > 1 || !row_lg || !wc) return fail(FFG_E_ARG, "geometry query");
    ffg_plan pl{};
    pl.lg = lg, pl.r3 = r3, pl.L = (uint64_t)(r3 ? 3 : 1) << lg, pl.split = 1; // split: always the four-step
    gpu_geometry(&pl);
    FourStep G = four_step_geometry(pl, true);
    *row_lg = pl.row_lg;
    *wc = G.wc;
    return FFG_OK;
}

extern "C" int ffg_load_tuning(const char *path) {
    std::lock_guard<std::recursive_mutex> lk(g_mu);
    FILE *f = path ? fopen(path, "r") : nullptr;
    if (!f) return fail(FFG_E_ARG, "tuning file %s", path ? path : "(null)");
    char word[32];
    std::vector<float> params;
    int rc = FFG_OK;
    while (rc == FFG_OK && fscanf(f, "%31s", word) == 1) {
        if (word[0] == '#') {
            int ch;
            while ((ch = fgetc(f)) != EOF && ch != '\n') {
            }
        } else if (!strcmp(word, "geometry")) {
            unsigned lg, r3, c, wc;
            if (fscanf(f, "%u %u %u %u", &lg, &r3, &c, &wc) != 4) rc = fail(FFG_E_ARG, "tuning: geometry line");
            else rc = ffg_set_geometry(lg, r3, c, wc);
        } else if (!strcmp(word, "mlp")) {
            unsigned n;
            if (fscanf(f, "%u", &n) != 1 || n != FFG_MLP_NPARAM) {
                rc = fail(FFG_E_ARG, "tuning: mlp needs %d parameters", FFG_MLP_NPARAM);
                break;
            }
            params.resize(n);
            for (unsigned i = 0; i < n && rc == FFG_OK; i++)
                if (fscanf(f, "%f", &params[i]) != 1) rc = fail(FFG_E_ARG, "tuning: mlp parameter %u", i);
        } else {
            rc = fail(FFG_E_ARG, "tuning: unknown entry %s", word);
        }
    }
    fclose(f);
    if (rc == FFG_OK && !params.empty()) rc = ffg_mlp_set(params.data());
    return rc;
}

// Words of the ticket pool that are not zero (all must be, between calls).
extern "C" int64_t ffg_tickets_in_use(void) {
    std::lock_guard<std::recursive_mutex> lk(g_mu);
    if (!g_tickets) return 0;
    cudaStreamSynchronize(g.stream);
    const size_t nt = (size_t)kTicketsLive + kTicketsCapture + 1;
    std::vector<uint32_t> h(nt);
    if (cudaMemcpy(h.data(), g_tickets, nt * 4, cudaMemcpyDeviceToHost)) return -1;
    int64_t c = 0;
    for (uint32_t v : h) c += v != 0;
    return c;
}

// ------------------------------------------------------------ fingerprints

static const uint64_t kFpPrimes[FFG_FP_PRIMES] = {18446744073709551557ull, 18446744073709551533ull,
                                                  9223372036854775783ull, 4611686018427387847ull};

// The fingerprint of x (device, n limbs) on stream st, scratch from the arena.
static int fingerprint_dev(const uint64_t *x, size_t n, uint64_t *out, cudaStream_t st) {
    uint64_t *partial = (uint64_t *)arena_alloc((size_t)fingerprint_blocks() * FFG_FP_PRIMES * 8);
    uint64_t *res = (uint64_t *)arena_alloc(8 * (FFG_FP_PRIMES + 2));
    if (!partial || !res) return fail(FFG_E_NOMEM, "device arena: fingerprint");
    unsigned long long *dbits = (unsigned long long *)(res + FFG_FP_PRIMES);
    CK(cudaMemsetAsync(dbits, 0, 8, st));
    cudaError_t e = launch_bits_mb(x, n, dbits, st);
    if (!e) e = launch_fingerprint(x, n, kFpPrimes, partial, ticket_get(), res, st);
    if (e) return fail(FFG_E_CUDA, "fingerprint: %s", cudaGetErrorString(e));
    uint64_t h[FFG_FP_PRIMES + 1], low = 0;
    CK(cudaMemcpyAsync(h, res, 8 * (FFG_FP_PRIMES + 1), cudaMemcpyDeviceToHost, st));
    if (n) CK(cudaMemcpyAsync(&low, x, 8, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    out[0] = h[FFG_FP_PRIMES];
    out[1] = low;
    for (int k = 0; k < FFG_FP_PRIMES; k++) out[2 + k] = h[k];
    return FFG_OK;
}

extern "C" int ffg_fingerprint_device(const uint64_t *x, size_t n, uint64_t *out) {
    std::lock_guard<std::recursive_mutex> lk(g_mu);
    int rc = ensure_ready();
    if (rc) return rc;
    if ((!x && n) || !out) return fail(FFG_E_ARG, "ffg_fingerprint_device arguments");
    CK(cudaStreamSynchronize(g.stream));
    arena_reset();
    return fingerprint_dev(x, n, out, g.stream);
}

extern "C" int ffg_fingerprint_host(const uint64_t *x, size_t n, uint64_t *out) {
    std::lock_guard<std::recursive_mutex> lk(g_mu);
    int rc = ensure_ready();
    if (rc) return rc;
    if ((!x && n) || !out) return fail(FFG_E_ARG, "ffg_fingerprint_host arguments");
    CK(cudaStreamSynchronize(g.stream));
    arena_reset();
    uint64_t *dx = (uint64_t *)arena_alloc(std::max<size_t>(1, n) * 8);
    if (!dx) return fail(FFG_E_NOMEM, "device arena: fingerprint input");
    if (n) CK(cudaMemcpyAsync(dx, x, n * 8, cudaMemcpyHostToDevice, g.stream));
    return fingerprint_dev(dx, n, out, g.stream);
}
