// Batches of independent products on the device (ffg_mul_batch_device /
// _host, ffg_time_batch): each product's method is resolved (the plain
// dispatch, a forced method, or the learned cost model), schoolbook products
// share one launch, products sharing an NTT plan share one launch set, and
// every CRT of the batch is one launch.  Also the cost model's C ABI (features,
// training, gradients, predictions, installed parameters).
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

// ------------------------------------------------------------ batches

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
int method_plan(int method, uint64_t bits_a, uint64_t bits_b, int square, BJob *j) {
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
void mlp_free() {
    if (g_mlp) cudaFree(g_mlp);
    g_mlp = nullptr;
}

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
// Streams a batch's plan groups run on besides the caller's (its lanes), with
// the events that fork them from and join them back to the caller's stream.
// FFG_BATCH_LANES sets the number of lanes, the caller's stream included
// (default 4; 1 runs every group on the caller's stream).
constexpr int kMaxLanes = 8;
static cudaStream_t g_lane[kMaxLanes - 1];
static cudaEvent_t g_fork = nullptr, g_join[kMaxLanes - 1];
static int g_lanes_made = 0;

static int batch_lanes() {
    static int v = -1;
    if (v < 0) {
        const char *e = getenv("FFG_BATCH_LANES");
        v = e && *e ? atoi(e) : 4;
        v = std::max(1, std::min(kMaxLanes, v));
    }
    return v;
}

// Side streams 1 .. n - 1 and their events, made once (before any capture).
static cudaError_t lanes_make(int n) {
    cudaError_t e = cudaSuccess;
    if (!g_fork && (e = cudaEventCreateWithFlags(&g_fork, cudaEventDisableTiming))) return e;
    for (; g_lanes_made < n - 1; g_lanes_made++) {
        if ((e = cudaStreamCreateWithFlags(&g_lane[g_lanes_made], cudaStreamNonBlocking))) return e;
        if ((e = cudaEventCreateWithFlags(&g_join[g_lanes_made], cudaEventDisableTiming))) return e;
    }
    return e;
}

void lanes_free() {
    for (int i = 0; i < g_lanes_made; i++) {
        cudaStreamDestroy(g_lane[i]);
        cudaEventDestroy(g_join[i]);
    }
    g_lanes_made = 0;
    if (g_fork) cudaEventDestroy(g_fork);
    g_fork = nullptr;
}

int run_batch(std::vector<BJob> &jobs, cudaStream_t st, cudaGraph_t *capture) {
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
    // The plan groups are independent until the CRTs: they run on lanes (the
    // caller's stream and side streams forked from it, joined back before the
    // CRT launch), so the launches of small groups, which leave most SMs idle,
    // overlap the large ones.  Groups go to the least loaded lane, largest
    // predicted cost first (count x L log L; the schoolbook launch by its
    // limb products).
    const int nlanes = std::min<int>(batch_lanes(), (int)launches.size() + (sj.empty() ? 0 : 1));
    std::vector<int> lane_of(launches.size(), 0);
    int school_lane = 0;
    if (nlanes > 1) {
        CK(lanes_make(nlanes));
        std::vector<std::pair<double, int>> order; // (cost, index; -1 the schoolbook launch)
        for (size_t i = 0; i < launches.size(); i++)
            order.push_back({(double)launches[i].count * (double)launches[i].pl.L * (launches[i].pl.lg + 2), (int)i});
        if (!sj.empty()) order.push_back({school_bytes * school_bytes / (64.0 * (double)sj.size()), -1});
        std::sort(order.begin(), order.end(), [](const auto &x, const auto &y) { return x.first > y.first; });
        std::vector<double> load(nlanes, 0.0);
        for (const auto &o : order) {
            const int l = (int)(std::min_element(load.begin(), load.end()) - load.begin());
            load[l] += o.first;
            if (o.second < 0) school_lane = l;
            else lane_of[o.second] = l;
        }
    }
    auto lane = [&](int l) { return l == 0 ? st : g_lane[l - 1]; };
    // with `capture`, the launches (not the job upload) become a CUDA graph
    // instead of running: the autotuner replays it to time the device alone
    if (capture) {
        if (!splits.empty()) return fail(FFG_E_ARG, "batch capture: split products allocate while running");
        CK(cudaStreamSynchronize(st));
        CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        g_capturing = true;
    }
    bool forked = false;
    auto join = [&]() -> cudaError_t {
        cudaError_t e = cudaSuccess;
        for (int l = 1; forked && l < nlanes && !e; l++) {
            e = cudaEventRecord(g_join[l - 1], lane(l));
            if (!e) e = cudaStreamWaitEvent(st, g_join[l - 1], 0);
        }
        forked = false;
        return e;
    };
    auto end_capture = [&](int rc) -> int {
        cudaError_t je = join();
        if (!rc && je) rc = fail(FFG_E_CUDA, "batch lanes: %s", cudaGetErrorString(je));
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
    if (nlanes > 1) {
        forked = true;
        e = cudaEventRecord(g_fork, st);
        for (int l = 1; l < nlanes && !e; l++) e = cudaStreamWaitEvent(lane(l), g_fork, 0);
        if (e) return end_capture(fail(FFG_E_CUDA, "batch lanes: %s", cudaGetErrorString(e)));
    }
    for (size_t base = 0; base < sj.size(); base += 65535) {
        const uint32_t cnt = (uint32_t)std::min<size_t>(65535, sj.size() - base);
        e = launch_school_batch((const SchoolJob *)(dimg + school_off) + base, cnt, school_ctas_max,
                                lane(school_lane), school_bytes * cnt / sj.size());
        if (e) return end_capture(fail(FFG_E_CUDA, "schoolbook batch: %s", cudaGetErrorString(e)));
    }
    for (size_t li = 0; li < launches.size(); li++) {
        const Launch &ln = launches[li];
        const cudaStream_t ls = lane(lane_of[li]);
        const bool sq = ln.key.square != 0;
        if (ln.key.kernel == 0) {
            ConvJobs cjs{};
            cjs.ext = (const ConvJob *)(dimg + ln.conv_off);
            e = launch_conv_small(g.P3, cjs, (uint32_t)ln.count, (uint32_t)ln.pl.L, !sq, ls, ln.conv_bytes);
            if (e) return end_capture(fail(FFG_E_CUDA, "batched one-CTA transforms: %s", cudaGetErrorString(e)));
        } else {
            FourStep G = four_step_geometry(ln.pl, sq);
            const size_t per = sq ? 65535 : 32767;
            for (size_t base = 0; base < ln.count; base += per) {
                FSJobs fjs{};
                fjs.ext = (const FSJob *)(dimg + ln.conv_off) + base;
                const uint32_t cnt = (uint32_t)std::min(per, ln.count - base);
                e = launch_four_step(g.P3, G, fjs, cnt, ls, ln.conv_bytes * cnt / ln.count);
                if (e) return end_capture(fail(FFG_E_CUDA, "batched four-step: %s", cudaGetErrorString(e)));
            }
        }
    }
    if ((e = join())) return end_capture(fail(FFG_E_CUDA, "batch lanes: %s", cudaGetErrorString(e)));
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

using namespace ffg;

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
