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
#include "ffg_internal.h"

namespace ffg {

typedef unsigned __int128 u128h;

static const uint32_t kP[3] = {2113929217u, 2013265921u, 1811939329u}; // src/ntt_arith.c:48-52
static const uint32_t kG[3] = {5u, 31u, 13u};
static int kMaxLg = 25; // NTT_MAX_LG (src/common.h:46-48); ffg_set_max_lg lowers it like -DNTT_MAX_LG
static const uint32_t kSmallMaxL = 4096;  // one-CTA transform up to this length for a single product
// The cost model's "kernel kind" feature keeps the bound it was trained with.
static const uint32_t kFeatureSmallL = 4096;
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

struct Block {
    char *ptr;
    size_t cap, used;
};

struct Ctx {
    bool ready = false;
    cudaStream_t stream = nullptr;
    Primes3 P3{};
    void *tables = nullptr;
    std::vector<Block> blocks;
    size_t max_L = 0;
    std::string err;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double chain_ms = 0;
    uint64_t chain_h2d = 0, chain_d2h = 0;
    int device = -1;
};

static Ctx g;
static std::recursive_mutex g_mu;
static void dec_free();

// ------------------------------------------------------------ ticket pool

// Zero words for the in-launch carry settle (see ticket_get in
// ffg_internal.h): the live region is handed out round-robin, captured
// launches take words of the capture region (a cached graph keeps its words
// while later work cycles through the live region), and the last word
// belongs to the allocation-free multiply.
constexpr uint32_t kTicketsLive = 1u << 16, kTicketsCapture = 1u << 13;
static uint32_t *g_tickets = nullptr;
// The decimal host entry point's device copy of its number, kept between calls.
static uint64_t *g_dec_in = nullptr;
static size_t g_dec_in_cap = 0;
static uint32_t g_ticket_live = 0, g_ticket_cap = 0;
static bool g_capturing = false, g_capture_starved = false;

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
static void ev_record(cudaEvent_t e, cudaStream_t st) {
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

static int fail(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g.err = buf;
    return code;
}

#define CK(call)                                                                                     \
    do {                                                                                             \
        cudaError_t e_ = (call);                                                                     \
        if (e_ != cudaSuccess) return fail(FFG_E_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                                           __FILE__, __LINE__);                                      \
    } while (0)

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

static int ensure_ready() {
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
static void arena_reset() {
    for (auto &b : g.blocks) b.used = 0;
}

// g_capturing is set while a stream capture is open: the arena must not grow
// then (no cudaMalloc may be issued); a request that would need a new block
// fails and the capture is abandoned.

static void *arena_alloc(size_t bytes) {
    bytes = (bytes + 255) & ~(size_t)255;
    for (auto &b : g.blocks)
        if (b.cap - b.used >= bytes) {
            void *p = b.ptr + b.used;
            b.used += bytes;
            return p;
        }
    if (g_capturing) {
        g_capture_starved = true;
        return nullptr;
    }
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
static uint64_t ntt_length(uint64_t conv, uint32_t *lg_out, uint32_t *r3_out) {
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
struct Geo {
    uint8_t set, c, wc;
};
static Geo g_geo[32][2];

// Shared memory of a four-step column tile (words) and row pass must fit one
// CTA; the radix-3 tables cover column lines 3 2^n with n < kR3TabLg.
static bool geo_valid(uint32_t lg, uint32_t r3, uint32_t c, uint32_t wc) {
    if (c < 4 || c > 13 || c > lg || wc < 8 || wc > 64 || (wc & (wc - 1)) || wc > (1u << c)) return false;
    const uint32_t rn = lg - c;
    if (rn < 2 || rn > (r3 ? (uint32_t)kR3TabLg - 1 : (uint32_t)FFG_LINE_LG)) return false;
    const uint32_t R = (r3 ? 3u : 1u) << rn;
    return (size_t)line_stride(R) * wc * 4 <= 200 * 1024;
}

static void gpu_geometry(ffg_plan *pl) {
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

static int plan_select(uint64_t bits_a, uint64_t bits_b, int square, ffg_plan *pl) {
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
static void scale_consts(uint64_t L, uint32_t *scl, uint32_t *scls) {
    for (int k = 0; k < 3; k++) {
        uint32_t p = kP[k];
        uint32_t v = mulm((uint32_t)((1ull << 32) % p), inv_mod((uint32_t)(L % p), p), p);
        scl[k] = v;
        scls[k] = shoup_q(v, p);
    }
}

// ---------------------------------------------------------------- multiply

struct Prod {
    const uint64_t *a, *b;
    uint64_t na, nb, bits_a, bits_b;
    uint64_t *out;   // na + nb + 1 limbs
    int64_t add;     // small constant added to the product
};

static FourStep four_step_geometry(const ffg_plan &pl, bool square) {
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
static int run_split(const Prod &pr, bool square, const ffg_plan &pl, cudaStream_t st) {
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

static uint64_t bits_of(const uint64_t *a, size_t n) {
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

static void chain_cache_clear() {
    for (auto &c : g_chains)
        if (c.exec) cudaGraphExecDestroy(c.exec);
    g_chains.clear();
}

// Results come back to the host in pinned buffers (a DMA straight into the
// caller's memory, no staging copy).  They are pooled: ffg_free / ffg_release
// return one to the pool, and the next result of a fitting size reuses it.
static std::vector<std::pair<void *, size_t>> g_pinned_out, g_pinned_pool;
static volatile size_t g_pinned_outstanding = 0;

static void *pinned_get(size_t bytes) {
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
static int pinned_release(void *p) {
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
            g_capture_starved = false;
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

// ------------------------------------------------------------ batches

// A product of a batch with its method resolved: schoolbook, or an NTT plan.
struct BJob {
    const uint64_t *a, *b;
    uint64_t na, nb, bits_a, bits_b;
    uint64_t *out;   // na + nb + 1 limbs on the device, fully written
    int square;
    int school;
    ffg_plan pl;
};

// The smallest lengths 2^k >= conv and 3 2^k >= conv (at least 16 and 48),
// as ntt_length (src/mul_ntt.c:78-93) spans them.
static void forced_lengths(uint64_t conv, uint64_t *Lp2, uint32_t *lgp2, uint64_t *Lr3, uint32_t *lgr3) {
    uint64_t L = 16;
    uint32_t lg = 4;
    while (L < conv) L <<= 1, lg++;
    uint64_t L3 = 48;
    uint32_t lg3 = 4;
    while (L3 < conv) L3 <<= 1, lg3++;
    *Lp2 = L, *lgp2 = lg, *Lr3 = L3, *lgr3 = lg3;
}

// The plan a method gives one product (methods: include/ffg.h FFG_M_*;
// FFG_M_LEARNED is resolved before this).
static int method_plan(int method, uint64_t bits_a, uint64_t bits_b, int square, BJob *j) {
    const uint64_t la = (bits_a + 63) / 64, lb = (bits_b + 63) / 64, minlen = la < lb ? la : lb;
    j->school = 0;
    if (method == FFG_M_PLAIN) {
        // the reference's thresholds (src/mul_basic.c:30-38, 64-106): schoolbook up to
        // 64 limbs; the NTT from 200; between them the reference recurses with
        // Karatsuba down to schoolbook products, which the GPU runs as one
        // schoolbook product
        method = minlen >= 200 ? FFG_M_NTT : FFG_M_SCHOOL;
    }
    if (method == FFG_M_SCHOOL) {
        j->school = 1;
        return FFG_OK;
    }
    int rc = plan_select(bits_a, bits_b, square, &j->pl);
    if (rc || j->pl.split || method == FFG_M_NTT) return rc;
    if (method != FFG_M_NTT_POW2 && method != FFG_M_NTT_R3) return fail(FFG_E_ARG, "unknown method %d", method);
    // the same width, the transform length forced to 2^k or 3 2^k
    ffg_plan q = j->pl;
    uint64_t Lp2, Lr3;
    uint32_t lgp2, lgr3;
    forced_lengths(q.conv, &Lp2, &lgp2, &Lr3, &lgr3);
    const uint64_t L = method == FFG_M_NTT_R3 ? Lr3 : Lp2;
    if (L > g.max_L) return FFG_OK; // past the cap: keep the reference's plan
    q.L = L, q.lg = method == FFG_M_NTT_R3 ? lgr3 : lgp2, q.r3 = method == FFG_M_NTT_R3;
    gpu_geometry(&q);
    j->pl = q;
    return FFG_OK;
}

// ------------------------------------------------------------ cost model

static float *g_mlp = nullptr;         // installed parameters on the device (FFG_MLP_NPARAM floats)
static std::vector<float> g_mlp_host;  // the installed parameters, uploaded on first use
static bool g_mlp_dirty = false;

// The installed model on the device (nullptr: none); uploads it after ffg_mlp_set.
static float *mlp_device() {
    if (g_mlp_host.empty()) return nullptr;
    if (g_mlp_dirty || !g_mlp) {
        if (!g_mlp && cudaMalloc(&g_mlp, FFG_MLP_NPARAM * sizeof(float)) != cudaSuccess) {
            g_mlp = nullptr;
            return nullptr;
        }
        if (cudaMemcpy(g_mlp, g_mlp_host.data(), FFG_MLP_NPARAM * sizeof(float), cudaMemcpyHostToDevice)) return nullptr;
        g_mlp_dirty = false;
    }
    return g_mlp;
}
static const float kLearnedMargin = 0.152f; // log2(1 / 0.9): a 10% predicted saving

// Features of a product: log2 limbs of the longer and shorter operand,
// squaring, log2 and radix of the reference plan's length, log2 of the
// forced 2^k and 3 2^k lengths, and whether the reference plan leaves the
// one-CTA kernel.  Lengths over 2^26 scale past 1.
static void mlp_features(uint64_t bits_a, uint64_t bits_b, int square, float *f) {
    if (square) bits_b = bits_a;
    const double la = std::log2((double)std::max<uint64_t>(1, (bits_a + 63) / 64));
    const double lb = std::log2((double)std::max<uint64_t>(1, (bits_b + 63) / 64));
    ffg_plan pl;
    plan_select(std::max<uint64_t>(1, bits_a), std::max<uint64_t>(1, bits_b), square, &pl);
    uint64_t Lp2, Lr3;
    uint32_t lgp2, lgr3;
    forced_lengths(pl.conv, &Lp2, &lgp2, &Lr3, &lgr3);
    f[0] = (float)(std::max(la, lb) / 20.0);
    f[1] = (float)(std::min(la, lb) / 20.0);
    f[2] = square ? 1.f : 0.f;
    f[3] = (float)(std::log2((double)pl.L) / 26.0);
    f[4] = pl.r3 ? 1.f : 0.f;
    f[5] = (float)(std::log2((double)Lp2) / 26.0);
    f[6] = (float)(std::log2((double)Lr3) / 26.0);
    f[7] = pl.split || pl.L > kFeatureSmallL ? 1.f : 0.f;
}

// Resolves FFG_M_LEARNED in meth[]: one inference launch over every such
// product, then per product the method of least predicted cost among those
// whose plan exists (the forced lengths within the cap).  Without a model,
// and for products the reference splits, the plain thresholds.
// The learned choice is a function of (bit lengths, squaring, transform cap)
// under the installed model: kept per shape, so a batch whose shapes were
// seen before needs no cost-model round trip (upload, inference, copy back,
// synchronize) before its first launch.  Cleared when the model changes.
struct LearnedKey {
    uint64_t ba, bb, cap;
    int sq;
    bool operator<(const LearnedKey &o) const { return std::tie(ba, bb, cap, sq) < std::tie(o.ba, o.bb, o.cap, o.sq); }
};
static std::map<LearnedKey, int> g_learned_memo;
static const size_t kLearnedMemoMax = 1 << 20;
// The last batch's shapes (a hash and the shapes themselves) and its
// resolved methods: a batch repeated call after call is resolved by one
// comparison pass, with no per-product lookups before its first launch.
static uint64_t g_learned_sig = 0, g_learned_cap = 0;
static std::vector<uint64_t> g_learned_shapes;
static std::vector<int> g_learned_meth;

static int learned_resolve_shapes(const uint64_t *ba, const uint64_t *bb, const int *sq, int *meth, size_t count,
                                  cudaStream_t st);

static int learned_resolve(const uint64_t *ba, const uint64_t *bb, const int *sq, int *meth, size_t count,
                           cudaStream_t st) {
    uint64_t h = 1469598103934665603ull ^ (uint64_t)g.max_L; // FNV-1a over the shapes and methods asked for
    for (size_t i = 0; i < count; i++) {
        h = (h ^ ba[i]) * 1099511628211ull;
        h = (h ^ bb[i]) * 1099511628211ull;
        h = (h ^ (uint64_t)(sq[i] ? 1 : 0) ^ ((uint64_t)(uint32_t)meth[i] << 8)) * 1099511628211ull;
    }
    if (h == g_learned_sig && g_learned_cap == (uint64_t)g.max_L && g_learned_meth.size() == count) {
        bool same = true;
        for (size_t i = 0; i < count && same; i++)
            same = g_learned_shapes[3 * i] == ba[i] && g_learned_shapes[3 * i + 1] == bb[i] &&
                   g_learned_shapes[3 * i + 2] == (((uint64_t)(uint32_t)meth[i] << 1) | (sq[i] ? 1u : 0u));
        if (same) {
            for (size_t i = 0; i < count; i++) meth[i] = g_learned_meth[i];
            return FFG_OK;
        }
    }
    g_learned_shapes.resize(3 * count);
    for (size_t i = 0; i < count; i++) {
        g_learned_shapes[3 * i] = ba[i];
        g_learned_shapes[3 * i + 1] = bb[i];
        g_learned_shapes[3 * i + 2] = ((uint64_t)(uint32_t)meth[i] << 1) | (sq[i] ? 1u : 0u);
    }
    g_learned_sig = 0;
    const int rc = learned_resolve_shapes(ba, bb, sq, meth, count, st);
    if (rc) return rc;
    g_learned_meth.assign(meth, meth + count);
    g_learned_sig = h;
    g_learned_cap = (uint64_t)g.max_L;
    return FFG_OK;
}

static int learned_resolve_shapes(const uint64_t *ba, const uint64_t *bb, const int *sq, int *meth, size_t count,
                                  cudaStream_t st) {
    std::vector<size_t> idx;
    for (size_t i = 0; i < count; i++) {
        if (meth[i] != FFG_M_LEARNED) continue;
        auto it = g_learned_memo.find(LearnedKey{ba[i], bb[i], (uint64_t)g.max_L, sq[i] ? 1 : 0});
        if (it != g_learned_memo.end()) meth[i] = it->second;
        else idx.push_back(i);
    }
    if (idx.empty()) return FFG_OK;
    float *model = mlp_device();
    if (!model) {
        if (!g_mlp_host.empty()) return fail(FFG_E_CUDA, "cost model upload");
        for (size_t i : idx) meth[i] = FFG_M_PLAIN;
        return FFG_OK;
    }
    std::vector<float> X(idx.size() * FFG_MLP_D), out(idx.size() * FFG_MLP_K);
    for (size_t k = 0; k < idx.size(); k++) mlp_features(ba[idx[k]], bb[idx[k]], sq[idx[k]], &X[k * FFG_MLP_D]);
    float *dX = (float *)arena_alloc(X.size() * sizeof(float)), *dO = (float *)arena_alloc(out.size() * sizeof(float));
    if (!dX || !dO) return fail(FFG_E_NOMEM, "device arena: cost model rows");
    CK(cudaMemcpyAsync(dX, X.data(), X.size() * sizeof(float), cudaMemcpyHostToDevice, st));
    cudaError_t e = launch_mlp_infer(model, dX, (uint32_t)idx.size(), dO, st);
    if (e) return fail(FFG_E_CUDA, "cost model inference: %s", cudaGetErrorString(e));
    CK(cudaMemcpyAsync(out.data(), dO, out.size() * sizeof(float), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    for (size_t k = 0; k < idx.size(); k++) {
        const size_t i = idx[k];
        ffg_plan pl;
        plan_select(std::max<uint64_t>(1, ba[i]), std::max<uint64_t>(1, bb[i]), sq[i], &pl);
        if (pl.split) {
            meth[i] = FFG_M_PLAIN;
            continue;
        }
        uint64_t Lp2, Lr3;
        uint32_t lgp2, lgr3;
        forced_lengths(pl.conv, &Lp2, &lgp2, &Lr3, &lgr3);
        // the plain thresholds judge: another method must be predicted at
        // least kLearnedMargin cheaper (log2 units) than the plain one
        const uint64_t minlen = std::min((ba[i] + 63) / 64, (bb[i] + 63) / 64);
        const int plain = minlen >= 200 ? FFG_M_NTT : FFG_M_SCHOOL;
        const float *o = &out[k * FFG_MLP_K];
        int best = plain;
        for (int m = 0; m < FFG_MLP_K; m++) {
            if ((m == FFG_M_NTT_POW2 && Lp2 > g.max_L) || (m == FFG_M_NTT_R3 && Lr3 > g.max_L)) continue;
            if (o[m] < o[best] && o[m] < o[plain] - kLearnedMargin) best = m;
        }
        meth[i] = best;
    }
    if (g_learned_memo.size() + idx.size() > kLearnedMemoMax) g_learned_memo.clear();
    for (size_t i : idx) g_learned_memo[LearnedKey{ba[i], bb[i], (uint64_t)g.max_L, sq[i] ? 1 : 0}] = meth[i];
    return FFG_OK;
}

struct GroupKey {
    uint32_t kernel, lg, r3, width, row_lg, square;
    bool operator<(const GroupKey &o) const {
        return std::tie(kernel, lg, r3, width, row_lg, square) < std::tie(o.kernel, o.lg, o.r3, o.width, o.row_lg, o.square);
    }
};

// longest line one CTA holds (FFG_LINE_LG); measured: with the fixed-shape
// four-step passes, groups of 64+ products up to this length still run
// faster as one CTA per product and prime (the decimal conversion of F(10^8):
// 14.2 ms, against 15.1 / 17.8 ms with the bound at 8192 / 4096)
static const uint64_t kBatchSmallMaxL = 16384;
static const size_t kBatchSmallMin = 64;       // products of one plan (a decimal level has hundreds)

// Runs a batch: one schoolbook launch for every schoolbook product, then per
// group of products sharing an NTT plan one transform launch set and one CRT
// launch; split products one by one.  Job records go to the device in one
// copy.
static int run_batch(std::vector<BJob> &jobs, cudaStream_t st, cudaGraph_t *capture = nullptr) {
    // Many products of one four-step plan up to L = kBatchSmallMaxL: one CTA
    // per (product, prime) holding the whole transform beats three launches
    // once the group alone fills the GPU (a doubling step's pair does not).
    {
        std::map<GroupKey, size_t> count;
        for (const BJob &J : jobs)
            if (!J.school && !J.pl.split && J.pl.kernel == 1 && J.pl.L <= kBatchSmallMaxL)
                count[GroupKey{1, J.pl.lg, J.pl.r3, J.pl.width, J.pl.row_lg, (uint32_t)J.square}]++;
        for (BJob &J : jobs)
            if (!J.school && !J.pl.split && J.pl.kernel == 1 && J.pl.L <= kBatchSmallMaxL &&
                count[GroupKey{1, J.pl.lg, J.pl.r3, J.pl.width, J.pl.row_lg, (uint32_t)J.square}] >= kBatchSmallMin) {
                J.pl.kernel = 0;
                J.pl.row_lg = 0;
            }
    }
    std::vector<SchoolJob> sj;
    std::map<GroupKey, std::vector<size_t>> groups;
    std::vector<size_t> splits;
    double school_bytes = 0;
    uint32_t school_ctas_max = 0;
    for (size_t i = 0; i < jobs.size(); i++) {
        BJob &J = jobs[i];
        if (J.school) {
            SchoolJob s{};
            s.a = J.a, s.b = J.square ? J.a : J.b;
            s.na = (J.bits_a + 63) / 64, s.nb = J.square ? s.na : (J.bits_b + 63) / 64;
            s.out = J.out;
            s.nlimbs = J.na + (J.square ? J.na : J.nb) + 1;
            s.maps = (uint32_t *)arena_alloc((size_t)school_ctas(s.nlimbs) * 4);
            if (!s.maps) return fail(FFG_E_NOMEM, "device arena: schoolbook maps");
            s.ticket = ticket_get();
            school_ctas_max = std::max(school_ctas_max, school_ctas(s.nlimbs));
            school_bytes += 8.0 * (double)(s.na + s.nb + s.nlimbs);
            sj.push_back(s);
        } else if (J.pl.split) {
            splits.push_back(i);
        } else {
            GroupKey k{J.pl.kernel, J.pl.lg, J.pl.r3, J.pl.width, J.pl.row_lg, (uint32_t)J.square};
            groups[k].push_back(i);
        }
    }
    // host images of every device job array, packed into one copy
    std::vector<char> img;
    auto put = [&](const void *p, size_t n) {
        size_t off = (img.size() + 255) & ~(size_t)255;
        img.resize(off + n);
        memcpy(img.data() + off, p, n);
        return off;
    };
    struct Launch {
        GroupKey key;
        size_t conv_off, count;
        double conv_bytes;
        ffg_plan pl;
    };
    std::vector<Launch> launches;
    // every group's CRTs, run after all transforms as one launch (k_crt_flat:
    // first[j] is the first CTA of CRT j)
    std::vector<CrtJob> crts;
    std::vector<uint32_t> crt_first{0};
    double crt_bytes = 0;
    size_t school_off = sj.empty() ? 0 : put(sj.data(), sj.size() * sizeof(SchoolJob));
    for (auto &kv : groups) {
        const GroupKey &k = kv.first;
        const ffg_plan &pl = jobs[kv.second[0]].pl;
        const uint64_t L = pl.L;
        const uint32_t w = pl.width;
        std::vector<ConvJob> cj;
        std::vector<FSJob> fj;
        uint32_t scl[3], scls[3];
        scale_consts(L, scl, scls);
        Launch ln{k, 0, kv.second.size(), 0, pl};
        for (size_t idx : kv.second) {
            BJob &J = jobs[idx];
            uint32_t *ya = (uint32_t *)arena_alloc(3 * L * sizeof(uint32_t));
            uint32_t *yb = J.square ? nullptr : (uint32_t *)arena_alloc(3 * L * sizeof(uint32_t));
            if (!ya || (!J.square && !yb)) return fail(FFG_E_NOMEM, "device arena: batch residues");
            const uint64_t ca = (J.bits_a + w - 1) / w, cb = J.square ? ca : (J.bits_b + w - 1) / w;
            const uint64_t nb = J.square ? J.na : J.nb;
            if (k.kernel == 0) {
                ConvJob c{};
                c.a = J.a, c.b = J.square ? J.a : J.b, c.na = J.na, c.nb = nb, c.ca = ca, c.cb = cb;
                c.y = ya, c.y_stride = L, c.L_words = (uint32_t)L, c.n = pl.lg, c.r3 = pl.r3, c.width = w;
                c.square = J.square, c.conv = (uint32_t)(ca + cb - 1);
                memcpy(c.scl, scl, sizeof scl);
                memcpy(c.scls, scls, sizeof scls);
                cj.push_back(c);
            } else {
                FSJob f{};
                f.a = J.a, f.b = J.square ? J.a : J.b, f.na = J.na, f.nb = nb, f.ca = ca, f.cb = cb;
                f.ya = ya, f.yb = yb, f.width = w;
                fj.push_back(f);
            }
            ln.conv_bytes += 8.0 * (double)(J.na + (J.square ? 0 : nb)) + 12.0 * (double)(ca + cb - 1);
            CrtJob r{};
            r.y = ya, r.y_stride = L, r.conv = ca + cb - 1, r.out = J.out, r.nlimbs = J.na + nb + 1, r.width = w;
            r.maps = (uint32_t *)arena_alloc((size_t)crt_ctas(r.nlimbs, w) * 4);
            if (!r.maps) return fail(FFG_E_NOMEM, "device arena: batch carry maps");
            r.ticket = ticket_get();
            crt_bytes += 12.0 * (double)r.conv + 8.0 * (double)r.nlimbs;
            crt_first.push_back(crt_first.back() + crt_ctas(r.nlimbs, w));
            crts.push_back(r);
        }
        ln.conv_off = k.kernel == 0 ? put(cj.data(), cj.size() * sizeof(ConvJob)) : put(fj.data(), fj.size() * sizeof(FSJob));
        launches.push_back(ln);
    }
    const size_t crt_off = crts.empty() ? 0 : put(crts.data(), crts.size() * sizeof(CrtJob));
    const size_t first_off = crts.empty() ? 0 : put(crt_first.data(), crt_first.size() * sizeof(uint32_t));
    char *dimg = nullptr;
    if (!img.empty()) {
        dimg = (char *)arena_alloc(img.size());
        if (!dimg) return fail(FFG_E_NOMEM, "device arena: batch job records");
        CK(cudaMemcpyAsync(dimg, img.data(), img.size(), cudaMemcpyHostToDevice, st));
    }
    // with `capture`, the launches (not the job upload) become a CUDA graph
    // instead of running: the autotuner replays it to time the device alone
    if (capture) {
        if (!splits.empty()) return fail(FFG_E_ARG, "batch capture: split products allocate while running");
        CK(cudaStreamSynchronize(st));
        CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        g_capturing = true;
    }
    auto end_capture = [&](int rc) -> int {
        if (!capture) return rc;
        g_capturing = false;
        cudaGraph_t gr = nullptr;
        cudaError_t ce = cudaStreamEndCapture(st, &gr);
        if (rc) {
            if (gr) cudaGraphDestroy(gr);
            return rc;
        }
        if (ce) return fail(FFG_E_CUDA, "batch capture: %s", cudaGetErrorString(ce));
        *capture = gr;
        return FFG_OK;
    };
    cudaError_t e;
    for (size_t base = 0; base < sj.size(); base += 65535) {
        const uint32_t cnt = (uint32_t)std::min<size_t>(65535, sj.size() - base);
        e = launch_school_batch((const SchoolJob *)(dimg + school_off) + base, cnt, school_ctas_max, st,
                                school_bytes * cnt / sj.size());
        if (e) return end_capture(fail(FFG_E_CUDA, "schoolbook batch: %s", cudaGetErrorString(e)));
    }
    for (const Launch &ln : launches) {
        const bool sq = ln.key.square != 0;
        if (ln.key.kernel == 0) {
            ConvJobs cjs{};
            cjs.ext = (const ConvJob *)(dimg + ln.conv_off);
            e = launch_conv_small(g.P3, cjs, (uint32_t)ln.count, (uint32_t)ln.pl.L, !sq, st, ln.conv_bytes);
            if (e) return end_capture(fail(FFG_E_CUDA, "batched one-CTA transforms: %s", cudaGetErrorString(e)));
        } else {
            FourStep G = four_step_geometry(ln.pl, sq);
            const size_t per = sq ? 65535 : 32767;
            for (size_t base = 0; base < ln.count; base += per) {
                FSJobs fjs{};
                fjs.ext = (const FSJob *)(dimg + ln.conv_off) + base;
                const uint32_t cnt = (uint32_t)std::min(per, ln.count - base);
                e = launch_four_step(g.P3, G, fjs, cnt, st, ln.conv_bytes * cnt / ln.count);
                if (e) return end_capture(fail(FFG_E_CUDA, "batched four-step: %s", cudaGetErrorString(e)));
            }
        }
    }
    if (!crts.empty()) {
        e = launch_crt_flat((const CrtJob *)(dimg + crt_off), (const uint32_t *)(dimg + first_off),
                            (uint32_t)crts.size(), crt_first.back(), st, crt_bytes);
        if (e) return end_capture(fail(FFG_E_CUDA, "batched CRT: %s", cudaGetErrorString(e)));
    }
    for (size_t idx : splits) {
        BJob &J = jobs[idx];
        Prod p{J.a, J.square ? J.a : J.b, J.na, J.square ? J.na : J.nb, J.bits_a, J.square ? J.bits_a : J.bits_b,
               J.out, 0};
        int rc = run_split(p, J.square != 0, J.pl, st);
        if (rc) return rc;
    }
    return end_capture(FFG_OK);
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
    if (g_mlp) cudaFree(g_mlp);
    g_mlp = nullptr;
    if (g_dec_in) cudaFree(g_dec_in);
    g_dec_in = nullptr;
    g_dec_in_cap = 0;
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

// One batch of device jobs on stream st (the arena is reset first); with
// capture, its launches are captured into a graph instead of run.
static int batch_device_core(ffg_job *jobs, size_t count, cudaStream_t st, cudaGraph_t *capture = nullptr) {
    arena_reset();
    std::vector<uint64_t> ba(count), bb(count);
    std::vector<int> sq(count), meth(count);
    for (size_t i = 0; i < count; i++) {
        ba[i] = jobs[i].bits_a;
        sq[i] = jobs[i].square != 0;
        bb[i] = sq[i] ? jobs[i].bits_a : jobs[i].bits_b;
        meth[i] = jobs[i].method;
    }
    int rc = learned_resolve(ba.data(), bb.data(), sq.data(), meth.data(), count, st);
    if (rc) return rc;
    std::vector<BJob> bj;
    bj.reserve(count);
    for (size_t i = 0; i < count; i++) {
        ffg_job &u = jobs[i];
        const uint64_t nb = u.square ? u.na : u.nb;
        if (ba[i] == 0 || bb[i] == 0) {
            CK(cudaMemsetAsync(u.out, 0, (u.na + nb + 1) * 8, st));
            continue;
        }
        BJob J{u.a, u.square ? u.a : u.b, u.na, nb, ba[i], bb[i], u.out, sq[i], 0, {}};
        rc = method_plan(meth[i], ba[i], bb[i], sq[i], &J);
        if (rc) return rc;
        bj.push_back(J);
    }
    return run_batch(bj, st, capture);
}

extern "C" int ffg_mul_batch_device(ffg_job *jobs, size_t count, void *stream) {
    std::lock_guard<std::recursive_mutex> lk(g_mu);
    int rc = ensure_ready();
    if (rc) return rc;
    if (!jobs && count) return fail(FFG_E_ARG, "jobs is NULL");
    cudaStream_t st = stream ? (cudaStream_t)stream : g.stream;
    CK(cudaStreamSynchronize(st));
    return batch_device_core(jobs, count, st);
}

extern "C" int ffg_time_batch(ffg_job *jobs, size_t count, int reps, double *ms) {
    std::lock_guard<std::recursive_mutex> lk(g_mu);
    int rc = ensure_ready();
    if (rc) return rc;
    if ((!jobs && count) || reps < 1 || !ms) return fail(FFG_E_ARG, "ffg_time_batch arguments");
    cudaStream_t st = g.stream;
    CK(cudaStreamSynchronize(st));
    // the batch's launches captured once and replayed: device time only
    // (plans and job uploads stay outside the clock)
    cudaGraph_t gr = nullptr;
    if ((rc = batch_device_core(jobs, count, st, &gr))) return rc;
    cudaGraphExec_t ex = nullptr;
    cudaError_t e = cudaGraphInstantiate(&ex, gr, 0);
    cudaGraphDestroy(gr);
    if (e) return fail(FFG_E_CUDA, "batch graph: %s", cudaGetErrorString(e));
    e = cudaGraphLaunch(ex, st); // warm-up
    if (!e) e = cudaEventRecord(g.ev0, st);
    for (int r = 0; r < reps && !e; r++) e = cudaGraphLaunch(ex, st);
    if (!e) e = cudaEventRecord(g.ev1, st);
    if (!e) e = cudaEventSynchronize(g.ev1);
    float t = 0;
    if (!e) e = cudaEventElapsedTime(&t, g.ev0, g.ev1);
    cudaGraphExecDestroy(ex);
    if (e) return fail(FFG_E_CUDA, "batch timing: %s", cudaGetErrorString(e));
    *ms = t / reps;
    return FFG_OK;
}

// Host-side copies of a batch, split over threads: jobs [j0, j1) in `parts`
// ranges of about equal bytes, fn(i) per job.
template <typename F>
static void par_jobs(size_t j0, size_t j1, const std::vector<uint64_t> &bytes_upto, F fn) {
    const size_t n = j1 - j0;
    const uint64_t total = bytes_upto[j1] - bytes_upto[j0];
    unsigned hw = std::thread::hardware_concurrency();
    unsigned parts = (unsigned)std::min<uint64_t>(std::min<size_t>(n, hw ? hw : 4), 1 + total / (1u << 20));
    if (parts > 16) parts = 16;
    if (parts <= 1) {
        for (size_t i = j0; i < j1; i++) fn(i);
        return;
    }
    std::vector<std::thread> th;
    size_t lo = j0;
    for (unsigned k = 1; k <= parts && lo < j1; k++) {
        const uint64_t goal = bytes_upto[j0] + total * k / parts;
        size_t hi = lo + 1;
        while (hi < j1 && bytes_upto[hi] < goal) hi++;
        if (k == parts) hi = j1;
        th.emplace_back([lo, hi, &fn] {
            for (size_t i = lo; i < hi; i++) fn(i);
        });
        lo = hi;
    }
    for (auto &t : th) t.join();
}

// ffg_mul_batch_host: the operands are staged into pinned memory by several
// threads, a slice of jobs at a time, each slice's host-to-device copy
// overlapping the staging of the next; the products come back the same way,
// a slice's device-to-host copy overlapping the unstaging of the one before.
extern "C" int ffg_mul_batch_host(ffg_job *jobs, size_t count) {
    std::lock_guard<std::recursive_mutex> lk(g_mu);
    int rc = ensure_ready();
    if (rc) return rc;
    if (!jobs && count) return fail(FFG_E_ARG, "jobs is NULL");
    cudaStream_t st = g.stream;
    CK(cudaStreamSynchronize(st));
    arena_reset();
    // normalized sizes, one staging image of every operand, one result area
    std::vector<uint64_t> na(count), nb(count), ba(count), bb(count), aoff(count + 1), boff(count), roff(count + 1);
    std::vector<uint64_t> in_upto(count + 1), out_upto(count + 1);
    uint64_t in_limbs = 0, out_limbs = 0;
    for (size_t i = 0; i < count; i++) {
        ffg_job &u = jobs[i];
        ba[i] = bits_of(u.a, u.na);
        bb[i] = u.square ? ba[i] : bits_of(u.b, u.nb);
        na[i] = std::max<uint64_t>(1, (ba[i] + 63) / 64);
        nb[i] = std::max<uint64_t>(1, (bb[i] + 63) / 64);
        aoff[i] = in_limbs;
        in_upto[i] = in_limbs * 8;
        in_limbs += na[i];
        boff[i] = u.square ? aoff[i] : in_limbs;
        if (!u.square) in_limbs += nb[i];
        roff[i] = out_limbs;
        out_upto[i] = out_limbs * 8;
        out_limbs += na[i] + nb[i] + 1;
    }
    aoff[count] = in_limbs, roff[count] = out_limbs;
    in_upto[count] = in_limbs * 8, out_upto[count] = out_limbs * 8;
    uint64_t *din = (uint64_t *)arena_alloc(std::max<uint64_t>(1, in_limbs) * 8);
    uint64_t *dout = (uint64_t *)arena_alloc(std::max<uint64_t>(1, out_limbs) * 8);
    if (!din || !dout) return fail(FFG_E_NOMEM, "device arena: batch operands");
    // staging buffers go back to the pool on every path, after the stream is idle
    struct Staging {
        void *p = nullptr;
        cudaStream_t st;
        ~Staging() {
            if (p) {
                cudaStreamSynchronize(st);
                pinned_release(p);
            }
        }
    } in_buf{nullptr, st}, out_buf{nullptr, st};
    uint64_t *hin = (uint64_t *)(in_buf.p = pinned_get(std::max<uint64_t>(1, in_limbs) * 8));
    uint64_t *hout = (uint64_t *)(out_buf.p = pinned_get(std::max<uint64_t>(1, out_limbs) * 8));
    if (!hin || !hout) return fail(FFG_E_NOMEM, "pinned staging");
    // slices of about 1/8 of the bytes each (whole jobs)
    auto slices = [&](const std::vector<uint64_t> &upto) {
        std::vector<size_t> cut{0};
        for (int k = 1; k < 8; k++) {
            size_t i = cut.back();
            while (i < count && upto[i] < upto[count] * k / 8) i++;
            if (i > cut.back()) cut.push_back(i);
        }
        if (cut.back() != count) cut.push_back(count);
        return cut;
    };
    const std::vector<size_t> icut = slices(in_upto);
    for (size_t k = 0; k + 1 < icut.size(); k++) {
        const size_t j0 = icut[k], j1 = icut[k + 1];
        par_jobs(j0, j1, in_upto, [&](size_t i) {
            memcpy(hin + aoff[i], jobs[i].a, std::min(na[i], jobs[i].na) * 8);
            if (na[i] > jobs[i].na) hin[aoff[i]] = 0;
            if (!jobs[i].square) {
                memcpy(hin + boff[i], jobs[i].b, std::min(nb[i], jobs[i].nb) * 8);
                if (nb[i] > jobs[i].nb) hin[boff[i]] = 0;
            }
        });
        CK(cudaMemcpyAsync(din + aoff[j0], hin + aoff[j0], (aoff[j1] - aoff[j0]) * 8, cudaMemcpyHostToDevice, st));
    }
    std::vector<int> sqv(count), meth(count);
    for (size_t i = 0; i < count; i++) sqv[i] = jobs[i].square != 0, meth[i] = jobs[i].method;
    if ((rc = learned_resolve(ba.data(), bb.data(), sqv.data(), meth.data(), count, st))) return rc;
    std::vector<BJob> bj;
    for (size_t i = 0; i < count; i++) {
        if (ba[i] == 0 || bb[i] == 0) {
            CK(cudaMemsetAsync(dout + roff[i], 0, (na[i] + nb[i] + 1) * 8, st));
            continue;
        }
        BJob J{din + aoff[i], din + boff[i], na[i], nb[i], ba[i], bb[i], dout + roff[i], jobs[i].square != 0, 0, {}};
        if ((rc = method_plan(meth[i], ba[i], bb[i], jobs[i].square != 0, &J))) return rc;
        bj.push_back(J);
    }
    if ((rc = run_batch(bj, st))) return rc;
    const std::vector<size_t> ocut = slices(out_upto);
    std::vector<cudaEvent_t> ev(ocut.size());
    for (auto &e : ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    struct Events {
        std::vector<cudaEvent_t> &v;
        ~Events() {
            for (auto e : v)
                if (e) cudaEventDestroy(e);
        }
    } ev_guard{ev};
    for (size_t k = 0; k + 1 < ocut.size(); k++) {
        const size_t j0 = ocut[k], j1 = ocut[k + 1];
        CK(cudaMemcpyAsync(hout + roff[j0], dout + roff[j0], (roff[j1] - roff[j0]) * 8, cudaMemcpyDeviceToHost, st));
        CK(cudaEventRecord(ev[k], st));
    }
    for (size_t k = 0; k + 1 < ocut.size(); k++) {
        CK(cudaEventSynchronize(ev[k]));
        par_jobs(ocut[k], ocut[k + 1], out_upto, [&](size_t i) {
            uint64_t n = na[i] + nb[i];
            while (n > 1 && hout[roff[i] + n - 1] == 0) n--;
            memcpy(jobs[i].out, hout + roff[i], n * 8);
            jobs[i].nout = n;
        });
    }
    return FFG_OK;
}

// ------------------------------------------------------------ cost model ABI

extern "C" int ffg_mlp_features(uint64_t bits_a, uint64_t bits_b, int square, float *f) {
    std::lock_guard<std::recursive_mutex> lk(g_mu);
    if (!f) return fail(FFG_E_ARG, "f is NULL");
    mlp_features(bits_a, bits_b, square, f);
    return FFG_OK;
}

// Device copies of rows (X, method, y) in the arena.
static int mlp_upload(const float *X, const int32_t *M, const float *Y, size_t n, float **dX, int32_t **dM, float **dY,
                      cudaStream_t st) {
    *dX = (float *)arena_alloc(std::max<size_t>(1, n) * FFG_MLP_D * sizeof(float));
    *dM = (int32_t *)arena_alloc(std::max<size_t>(1, n) * sizeof(int32_t));
    *dY = (float *)arena_alloc(std::max<size_t>(1, n) * sizeof(float));
    if (!*dX || !*dM || !*dY) return fail(FFG_E_NOMEM, "device arena: training rows");
    for (size_t i = 0; i < n; i++)
        if (M[i] < 0 || M[i] >= FFG_MLP_K) return fail(FFG_E_ARG, "row %zu: method %d", i, (int)M[i]);
    if (n) {
        CK(cudaMemcpyAsync(*dX, X, n * FFG_MLP_D * sizeof(float), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(*dM, M, n * sizeof(int32_t), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(*dY, Y, n * sizeof(float), cudaMemcpyHostToDevice, st));
    }
    return FFG_OK;
}

extern "C" int ffg_mlp_train(float *params, const float *X, const int32_t *method, const float *y, size_t n, int epochs,
                             float lr, float *loss_hist) {
    std::lock_guard<std::recursive_mutex> lk(g_mu);
    int rc = ensure_ready();
    if (rc) return rc;
    if (!params || (!n && epochs > 0) || epochs < 0 || (n && (!X || !method || !y)))
        return fail(FFG_E_ARG, "ffg_mlp_train arguments");
    cudaStream_t st = g.stream;
    CK(cudaStreamSynchronize(st));
    arena_reset();
    float *dX, *dY;
    int32_t *dM;
    if ((rc = mlp_upload(X, method, y, n, &dX, &dM, &dY, st))) return rc;
    float *dP = (float *)arena_alloc(FFG_MLP_NPARAM * sizeof(float));
    float *dL = (float *)arena_alloc(std::max(1, epochs) * sizeof(float));
    if (!dP || !dL) return fail(FFG_E_NOMEM, "device arena: parameters");
    CK(cudaMemcpyAsync(dP, params, FFG_MLP_NPARAM * sizeof(float), cudaMemcpyHostToDevice, st));
    cudaError_t e = launch_mlp_train(dP, dX, dM, dY, (uint32_t)n, (uint32_t)epochs, lr, dL, st);
    if (e) return fail(FFG_E_CUDA, "cost model training: %s", cudaGetErrorString(e));
    CK(cudaMemcpyAsync(params, dP, FFG_MLP_NPARAM * sizeof(float), cudaMemcpyDeviceToHost, st));
    if (loss_hist && epochs > 0) CK(cudaMemcpyAsync(loss_hist, dL, epochs * sizeof(float), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return FFG_OK;
}

extern "C" int ffg_mlp_grad(const float *params, const float *X, const int32_t *method, const float *y, size_t n,
                            float *grad, float *loss) {
    std::lock_guard<std::recursive_mutex> lk(g_mu);
    int rc = ensure_ready();
    if (rc) return rc;
    if (!params || !grad || !loss || !n || !X || !method || !y) return fail(FFG_E_ARG, "ffg_mlp_grad arguments");
    cudaStream_t st = g.stream;
    CK(cudaStreamSynchronize(st));
    arena_reset();
    float *dX, *dY;
    int32_t *dM;
    if ((rc = mlp_upload(X, method, y, n, &dX, &dM, &dY, st))) return rc;
    float *dP = (float *)arena_alloc(2 * FFG_MLP_NPARAM * sizeof(float) + 256), *dG = dP + FFG_MLP_NPARAM;
    float *dL = (float *)arena_alloc(sizeof(float));
    if (!dP || !dL) return fail(FFG_E_NOMEM, "device arena: parameters");
    CK(cudaMemcpyAsync(dP, params, FFG_MLP_NPARAM * sizeof(float), cudaMemcpyHostToDevice, st));
    cudaError_t e = launch_mlp_grad(dP, dX, dM, dY, (uint32_t)n, dG, dL, st);
    if (e) return fail(FFG_E_CUDA, "cost model gradient: %s", cudaGetErrorString(e));
    CK(cudaMemcpyAsync(grad, dG, FFG_MLP_NPARAM * sizeof(float), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(loss, dL, sizeof(float), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return FFG_OK;
}

extern "C" int ffg_mlp_predict(const float *params, const float *X, size_t n, float *out) {
    std::lock_guard<std::recursive_mutex> lk(g_mu);
    int rc = ensure_ready();
    if (rc) return rc;
    if ((!params && g_mlp_host.empty()) || (n && (!X || !out))) return fail(FFG_E_ARG, "ffg_mlp_predict arguments");
    cudaStream_t st = g.stream;
    CK(cudaStreamSynchronize(st));
    arena_reset();
    float *dX = (float *)arena_alloc(std::max<size_t>(1, n) * FFG_MLP_D * sizeof(float));
    float *dO = (float *)arena_alloc(std::max<size_t>(1, n) * FFG_MLP_K * sizeof(float));
    float *dP = params ? (float *)arena_alloc(FFG_MLP_NPARAM * sizeof(float)) : mlp_device();
    if (!dX || !dO || !dP) return fail(FFG_E_NOMEM, "device arena: cost model rows");
    if (params) CK(cudaMemcpyAsync(dP, params, FFG_MLP_NPARAM * sizeof(float), cudaMemcpyHostToDevice, st));
    if (n) CK(cudaMemcpyAsync(dX, X, n * FFG_MLP_D * sizeof(float), cudaMemcpyHostToDevice, st));
    cudaError_t e = launch_mlp_infer(dP, dX, (uint32_t)n, dO, st);
    if (e) return fail(FFG_E_CUDA, "cost model inference: %s", cudaGetErrorString(e));
    if (n) CK(cudaMemcpyAsync(out, dO, n * FFG_MLP_K * sizeof(float), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return FFG_OK;
}

extern "C" int ffg_mlp_set(const float *params) {
    std::lock_guard<std::recursive_mutex> lk(g_mu);
    g_learned_memo.clear();
    g_learned_sig = 0;
    g_learned_meth.clear();
    if (!params) {
        g_mlp_host.clear();
        return FFG_OK;
    }
    g_mlp_host.assign(params, params + FFG_MLP_NPARAM);
    g_mlp_dirty = true;
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

// =================================================== decimal conversion
//
// big_to_string (src/decimal.c:229-281) on the device, breadth first.  With
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

namespace ffg {

// Leaves: pieces below 10^(19 2^(kDecLeafLg + 1)) = 10^2432 (at most 128 limbs),
// one thread each.  The reference stops its recursion two levels lower
// (DEC_LEAF_LG = 4, src/decimal.c); here the two lowest levels would hold tens
// of thousands of pieces whose job records cost more host time than their
// arithmetic costs the GPU.
static const int kDecLeafLg = 6;
static const uint64_t kDec19 = 10000000000000000000ull;

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

static void dec_free() {
    for (auto &L : g_dec) {
        if (L.P) cudaFree(L.P);
        if (L.m) cudaFree(L.m);
    }
    g_dec.clear();
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
