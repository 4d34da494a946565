// Host-side state and helpers shared by the host translation units of the GPU
// layer:
//   ffg_host.cu      the context, tables, device arena, pinned pool, plans,
//                    the multiply, the doubling chain and their C ABI;
//   ffg_batch.cu     batches of independent products, the cost model and the
//                    learned dispatch, and their C ABI;
//   ffg_dec_host.cu  the decimal conversion driver and its C ABI.
// Every C ABI entry point holds g_mu for its whole call: the context, its
// stream, its arena and its ticket pool are one per process (one device), and
// a call owns them until it returns.  Several devices or ranks are one process
// each.
#pragma once
#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "ffg.h"
#include "ffg_internal.h"

namespace ffg {

// The cost model's "kernel kind" feature keeps the one-CTA bound it was
// trained with.
constexpr uint32_t kFeatureSmallL = 4096;

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

extern Ctx g;
extern std::recursive_mutex g_mu;
// Set while a graph capture is open: launches then take capture tickets.
extern bool g_capturing;

// Records message fmt as the last error and returns code.
int fail(int code, const char *fmt, ...);

#define CK(call)                                                                                     \
    do {                                                                                             \
        cudaError_t e_ = (call);                                                                     \
        if (e_ != cudaSuccess) return fail(FFG_E_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                                           __FILE__, __LINE__);                                      \
    } while (0)

// Device, stream and tables ready (ffg_init with the default size if needed).
int ensure_ready();
// Device arena: every call resets it first; allocations are 256-byte aligned
// and live until the next reset.
void arena_reset();
void *arena_alloc(size_t bytes);
// Pinned host buffers handed to callers (released by ffg_release) or reused.
void *pinned_get(size_t bytes);
int pinned_release(void *p);
// An event record on st from the pool (profiling and timing).
void ev_record(cudaEvent_t e, cudaStream_t st);
// Bit length of a (n limbs, host).
uint64_t bits_of(const uint64_t *a, size_t n);
// Drops the cached doubling-chain graphs.
void chain_cache_clear();

// ------------------------------------------------------------------- plans

// A tuned four-step geometry per (log2 length, radix-3 flag), set by
// ffg_set_geometry: row length 2^c and column-tile width wc.
struct Geo {
    uint8_t set, c, wc;
};
extern Geo g_geo[32][2];
bool geo_valid(uint32_t lg, uint32_t r3, uint32_t c, uint32_t wc);
// Fills the GPU kernel geometry (kernel kind, row length, tile width) of pl.
void gpu_geometry(ffg_plan *pl);
// The smallest supported length 3^r3 2^lg >= conv.
uint64_t ntt_length(uint64_t conv, uint32_t *lg_out, uint32_t *r3_out);
// The reference's width/length plan of a product of the given bit lengths.
int plan_select(uint64_t bits_a, uint64_t bits_b, int square, ffg_plan *pl);
// 2^32 / L mod p per prime (Shoup pairs): the inverse transform's scale.
void scale_consts(uint64_t L, uint32_t *scl, uint32_t *scls);

// One product on the device.
struct Prod {
    const uint64_t *a, *b;
    uint64_t na, nb, bits_a, bits_b;
    uint64_t *out;   // na + nb + 1 limbs
    int64_t add;     // small constant added to the product
};
FourStep four_step_geometry(const ffg_plan &pl, bool square);
// The split multiply of one product past the largest transform.
int run_split(const Prod &pr, bool square, const ffg_plan &pl, cudaStream_t st);

// ---------------------------------------------------------------- batches

// A product of a batch with its method resolved: schoolbook, or an NTT plan.
struct BJob {
    const uint64_t *a, *b;
    uint64_t na, nb, bits_a, bits_b;
    uint64_t *out;   // na + nb + 1 limbs on the device, fully written
    int square;
    int school;
    ffg_plan pl;
};
// Resolves method (FFG_M_*) for one product into j's plan.
int method_plan(int method, uint64_t bits_a, uint64_t bits_b, int square, BJob *j);
// Runs a batch on stream st (launches grouped by plan); with capture, the
// launches are captured into *capture instead.
int run_batch(std::vector<BJob> &jobs, cudaStream_t st, cudaGraph_t *capture = nullptr);
// Frees the cost model's device parameters.
void mlp_free();
// Destroys the batches' side streams and their events.
void lanes_free();

// ---------------------------------------------------------------- decimal

// Frees the decimal conversion's cached powers, reciprocals and input copy.
void dec_free();

} // namespace ffg
