// SPDX-License-Identifier: Apache-2.0
//
// Host orchestration and C ABI of the B200 compact encoder.
//
// One call: plan on the host (closed-form layout, a few KB) -> prologue
// kernel (zero status, header bytes) -> level kernels for the levels whose
// nodes exceed a tile -> one tile kernel finishing every subtree in shared
// memory.  Everything runs on one stream; scratch lives in a pooled
// per-device workspace so repeated calls allocate nothing.
#include "../../include/benes_b200.h"
#include "batch_levels.cuh"
#include "kernels.cuh"
#include "layout.hpp"
#include "plan.hpp"
#include "tile.cuh"
#include "walk.cuh"

#include <cuda_runtime.h>
#include <dlfcn.h>
#include <immintrin.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

namespace bpb200 {
namespace {

constexpr uint64_t kTileMaxEntries = 8192;
constexpr uint32_t kTileSmemBudget = 224 * 1024;
// Above this a tile runs as one 1024-thread CTA per SM (tile_encode_wide).
constexpr uint32_t kTileSmemTwoPerSm = 112 * 1024;
constexpr int kLevelThreads = 256;

// Kernel kinds reported by bpb200_last_profile.
enum KernelKind : int {
    kKindPrologue = 0,
    kKindInverse,
    kKindDescriptors,
    kKindUnion,
    kKindOrient,
    kKindResolve,
    kKindOutputBits,
    kKindTile,
    kKindEmit,
    kKindWalk,
    kKindJump,
    kKindPlace, // partitioned inverse (level_bucket + level_place)
    kKernelKinds
};

struct CudaFail {
    cudaError_t err;
    const char* what;
};

void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        throw CudaFail{e, what};
    }
}

// ------------------------------------------------------------ workspace

struct Workspace {
    int device = -1;
    cudaStream_t stream = nullptr;
    cudaStream_t copy_stream = nullptr; // early blob download of the host path
    cudaEvent_t start = nullptr, stop = nullptr;
    cudaEvent_t early = nullptr;        // the blob's first cluster groups are final
    cudaEvent_t parts[8] = {};          // tile parts done (progressive blob download)
    cudaEvent_t inparts[8] = {};        // input parts on the device (host path upload)
    Plan* d_plan = nullptr;
    Plan* h_plan = nullptr;       // pinned staging for the plan upload
    uint32_t* d_status = nullptr;
    uint32_t* h_status = nullptr; // pinned
    uint32_t* vals[2] = {nullptr, nullptr};
    uint32_t* inv = nullptr;
    uint32_t* inv2 = nullptr;     // next level's inverse (levels alternate the two)
    uint32_t* uf = nullptr;
    uint32_t* xbits = nullptr;
    uint32_t* ybits = nullptr;
    uint32_t* owner = nullptr;             // ruler id stamped on each walked even vertex, per pair-node
    uint4* state[2] = {nullptr, nullptr};  // ruler states; [1] holds the super-ruler states
    uint32_t* super_of = nullptr;          // super-ruler (or stamped colour) of each ruler
    uint32_t* control = nullptr;           // per-level control words (walk.cuh)
    uint2* records = nullptr;              // partitioned-inverse records (kernels.cuh)
    uint32_t* cursor = nullptr;            // fill level of each destination window
    NodeAddress* addr[2] = {nullptr, nullptr};
    uint64_t slot_cap = 0, pair_cap = 0, node_cap = 0;
    void* input = nullptr;        // staging for host-path inputs
    uint64_t input_cap = 0;
    uint32_t* blob = nullptr;     // staging for host-path blobs
    uint64_t blob_cap = 0;
    std::vector<cudaEvent_t> events; // profiling events, reused across calls
    bool busy = false;

    void release_scratch() {
        for (void* p : {(void*)vals[0], (void*)vals[1], (void*)inv, (void*)inv2, (void*)uf,
                 (void*)xbits,
                 (void*)ybits, (void*)owner, (void*)state[0], (void*)state[1], (void*)super_of,
                 (void*)control,
                 (void*)records, (void*)cursor, (void*)addr[0], (void*)addr[1]}) {
            if (p) cudaFree(p);
        }
        vals[0] = vals[1] = inv = inv2 = uf = xbits = ybits = owner = control = cursor = nullptr;
        super_of = nullptr;
        records = nullptr;
        state[0] = state[1] = nullptr;
        addr[0] = addr[1] = nullptr;
        slot_cap = pair_cap = node_cap = 0;
    }
    void destroy() {
        release_scratch();
        if (input) cudaFree(input);
        if (blob) cudaFree(blob);
        if (d_plan) cudaFree(d_plan);
        if (d_status) cudaFree(d_status);
        if (h_plan) cudaFreeHost(h_plan);
        if (h_status) cudaFreeHost(h_status);
        if (start) cudaEventDestroy(start);
        if (stop) cudaEventDestroy(stop);
        if (early) cudaEventDestroy(early);
        for (cudaEvent_t e : parts) {
            if (e) cudaEventDestroy(e);
        }
        for (cudaEvent_t e : inparts) {
            if (e) cudaEventDestroy(e);
        }
        if (stream) cudaStreamDestroy(stream);
        if (copy_stream) cudaStreamDestroy(copy_stream);
        for (cudaEvent_t e : events) cudaEventDestroy(e);
        *this = Workspace();
    }
};

std::mutex g_pool_mutex;
std::vector<std::unique_ptr<Workspace>> g_pool;

Workspace* acquire(int device) {
    std::lock_guard<std::mutex> lock(g_pool_mutex);
    for (auto& w : g_pool) {
        if (!w->busy && w->device == device) {
            w->busy = true;
            return w.get();
        }
    }
    auto w = std::make_unique<Workspace>();
    w->device = device;
    check(cudaStreamCreateWithFlags(&w->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    check(cudaEventCreate(&w->start), "cudaEventCreate");
    check(cudaEventCreate(&w->stop), "cudaEventCreate");
    check(cudaStreamCreateWithFlags(&w->copy_stream, cudaStreamNonBlocking), "cudaStreamCreate");
    check(cudaEventCreateWithFlags(&w->early, cudaEventDisableTiming), "cudaEventCreate");
    for (cudaEvent_t& e : w->parts) {
        check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
    }
    for (cudaEvent_t& e : w->inparts) {
        check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
    }
    check(cudaMalloc(&w->d_plan, sizeof(Plan)), "cudaMalloc(plan)");
    check(cudaMallocHost(&w->h_plan, sizeof(Plan)), "cudaMallocHost(plan)");
    check(cudaMalloc(&w->d_status, sizeof(uint32_t)), "cudaMalloc(status)");
    check(cudaMallocHost(&w->h_status, sizeof(uint32_t)), "cudaMallocHost(status)");
    w->busy = true;
    g_pool.push_back(std::move(w));
    return g_pool.back().get();
}

void release(Workspace* w) {
    std::lock_guard<std::mutex> lock(g_pool_mutex);
    w->busy = false;
}

struct Lease {
    Workspace* w;
    explicit Lease(int device) : w(acquire(device)) {}
    ~Lease() { release(w); }
};

// Grows the level scratch to fit `p`.  Growth at least doubles the previous
// capacities: freeing device memory synchronises the whole device, so a
// workspace that serves requests of varying sizes (the batched and serving
// forms) must reach its final size after a few calls, not one per call.
void ensure_scratch(Workspace& w, const Plan& p) {
    uint64_t slots = p.tile_level > 0 ? p.max_slots : 0;
    uint64_t pairs = p.tile_level > 0 ? p.max_pairs : 0;
    uint64_t nodes = p.tile_level > 0 ? (1ull << (p.tile_level - 1)) : 0;
    const bool need_records = p.levels[0].cap > kWalkMaxNode;
    if (slots <= w.slot_cap && pairs <= w.pair_cap && nodes <= w.node_cap &&
        (w.records != nullptr || !need_records)) {
        return;
    }
    if (slots == 0) {
        return;
    }
    slots = std::max(slots, 2 * w.slot_cap);
    pairs = std::max(pairs, 2 * w.pair_cap);
    nodes = std::max(nodes, 2 * w.node_cap);
    w.release_scratch();
    check(cudaMalloc(&w.vals[0], slots * 4), "cudaMalloc(level array)");
    check(cudaMalloc(&w.vals[1], slots * 4), "cudaMalloc(level array)");
    check(cudaMalloc(&w.inv, slots * 4), "cudaMalloc(inverse)");
    check(cudaMalloc(&w.inv2, slots * 4), "cudaMalloc(inverse)");
    check(cudaMalloc(&w.uf, pairs * 4), "cudaMalloc(union-find)");
    check(cudaMalloc(&w.xbits, ((pairs + 31) / 32 + 1) * 4), "cudaMalloc(colour bits)");
    check(cudaMalloc(&w.ybits, ((pairs + 31) / 32 + 1) * 4), "cudaMalloc(output bits)");
    check(cudaMalloc(&w.owner, pairs * 4), "cudaMalloc(owners)"); // one per pair-node
    const uint64_t buckets = (slots >> kRulerLog2) + 1;
    check(cudaMalloc(&w.state[0], buckets * sizeof(uint4)), "cudaMalloc(ruler state)");
    check(cudaMalloc(&w.state[1], buckets * sizeof(uint4)), "cudaMalloc(ruler state)");
    check(cudaMalloc(&w.super_of, buckets * 4), "cudaMalloc(super rulers)");
    check(cudaMalloc(&w.control, kCtlWords * 4), "cudaMalloc(control)");
    if (p.levels[0].cap > kWalkMaxNode) {
        // only levels with nodes above L2 size use the partitioned inverse
        check(cudaMalloc(&w.records, slots * sizeof(uint2)), "cudaMalloc(records)");
        check(cudaMalloc(&w.cursor, kMaxWindows * 4), "cudaMalloc(cursors)");
    }
    check(cudaMalloc(&w.addr[0], nodes * sizeof(NodeAddress)), "cudaMalloc(descriptors)");
    check(cudaMalloc(&w.addr[1], nodes * sizeof(NodeAddress)), "cudaMalloc(descriptors)");
    w.slot_cap = slots;
    w.pair_cap = pairs;
    w.node_cap = nodes;
}

// ------------------------------------------------------------ prologue

struct Header {
    uint32_t bytes;
    uint8_t data[84];
};

__global__ void prologue(uint32_t* status, uint32_t* blob, Header h) {
    if (threadIdx.x == 0) {
        *status = 0;
    }
    // the header ends before the first section bit; only whole header bytes
    // are written, so it cannot clobber section bits sharing its last word
    uint8_t* b = reinterpret_cast<uint8_t*>(blob);
    for (uint32_t i = threadIdx.x; i < h.bytes; i += blockDim.x) {
        b[i] = h.data[i];
    }
}

// ------------------------------------------------------------ tile sizing

TileShape tile_shape(const Plan& p, uint32_t t0) {
    uint64_t slots = 0, pairs = 0;
    for (uint32_t l = t0; l <= p.depth; ++l) {
        const uint64_t n = 1ull << (l - t0);
        slots = std::max<uint64_t>(slots, n * p.levels[l].cap);
        pairs = std::max<uint64_t>(pairs, n * p.levels[l].pcap);
    }
    TileShape s;
    s.slots = (uint32_t)std::min<uint64_t>(slots, 1u << 30);
    s.pairs = (uint32_t)std::min<uint64_t>(pairs, 1u << 30);
    uint32_t off[9];
    s.smem = tile_smem_layout(s.slots, s.pairs, off);
    if (slots >= 65536 || pairs >= (1u << 30)) {
        s.smem = UINT32_MAX;
    }
    return s;
}

// Picks the tile level: the first level whose nodes fit `tile_max` entries
// and whose deepest padded tile level also fits the shared-memory budget.
void choose_tile(Plan& p, TileShape* shape, uint64_t tile_max = kTileMaxEntries) {
    uint32_t t0 = 0;
    while (t0 < p.depth && p.levels[t0].cap > tile_max) {
        ++t0;
    }
    TileShape s = tile_shape(p, t0);
    while (s.smem > kTileSmemBudget && t0 < p.depth) {
        ++t0;
        s = tile_shape(p, t0);
    }
    p.tile_level = t0;
    uint64_t slots = 0, pairs = 0;
    for (uint32_t l = 0; l <= t0; ++l) {
        slots = std::max<uint64_t>(slots, (1ull << l) * p.levels[l].cap);
        pairs = std::max<uint64_t>(pairs, (1ull << l) * p.levels[l].pcap);
    }
    p.max_slots = slots;
    p.max_pairs = pairs;
    *shape = s;
}

std::atomic<int> g_force_union_find{0};

// ------------------------------------------------------------ tuning
//
// Launch choices that change speed but never bytes, per size class (the
// class of a permutation of n entries is ceil(log2 n)):
//   walk_blocks_per_sm  persistent level_walk blocks per SM; resident
//                       walkers times the slots per ruler is the address
//                       window the walks keep live, which must stay in L2
//   walk_max_log2       largest node coloured by orbit walks (larger nodes
//                       by union-find); at most the compiled walk limit
//   jump_block_log2     largest super-ruler count whose pointer-jumping
//                       rounds run inside one CTA (else one launch pair per
//                       round)
//   tile_max_log2       largest node handed to the shared-memory tile
// The table comes from tuning.json beside this library (written by
// benes_perm_b200/tune.py; BPB200_TUNING_FILE names another file, "none"
// disables it), loaded once; classes it lacks take the nearest class it
// has, and without a table the compiled defaults apply.
// BPB200_WALK_BLOCKS_PER_SM overrides the default walk blocks per SM.
struct Tuning {
    uint32_t walk_blocks_per_sm;
    uint32_t walk_max_log2;
    uint32_t jump_block_log2;
    uint32_t tile_max_log2;
};

Tuning default_tuning() {
    static const Tuning t = [] {
        const char* env = std::getenv("BPB200_WALK_BLOCKS_PER_SM");
        const int v = env ? std::atoi(env) : 4;
        return Tuning{(uint32_t)(v < 1 ? 1 : (v > 8 ? 8 : v)), BPB200_WALK_MAX_LOG2,
            BPB200_JUMP_BLOCK_LOG2, 13};
    }();
    return t;
}

Tuning clamp_tuning(Tuning t) {
    auto clamp = [](uint32_t v, uint32_t lo, uint32_t hi) { return v < lo ? lo : (v > hi ? hi : v); };
    t.walk_blocks_per_sm = clamp(t.walk_blocks_per_sm, 1, 8);
    t.walk_max_log2 = clamp(t.walk_max_log2, 10, BPB200_WALK_MAX_LOG2);
    t.jump_block_log2 = clamp(t.jump_block_log2, 4, 18);
    t.tile_max_log2 = clamp(t.tile_max_log2, 9, 14);
    return t;
}

struct TuningTable {
    bool has[64] = {};
    Tuning at[64];
};

// Reads {"classes": {"<class>": {"<knob>": <int>, ...}, ...}}; anything
// else in the file is ignored.  A missing or malformed file gives an empty
// table.
TuningTable load_tuning_table() {
    TuningTable t;
    std::string path;
    if (const char* env = std::getenv("BPB200_TUNING_FILE")) {
        path = env;
    } else {
        Dl_info info{};
        if (dladdr((void*)&default_tuning, &info) != 0 && info.dli_fname != nullptr) {
            path = info.dli_fname;
            const size_t slash = path.find_last_of('/');
            path = (slash == std::string::npos ? std::string(".") : path.substr(0, slash)) +
                "/tuning.json";
        }
    }
    if (path.empty() || path == "none") return t;
    FILE* f = std::fopen(path.c_str(), "rb");
    if (f == nullptr) return t;
    std::string text;
    char buf[4096];
    size_t got;
    while ((got = std::fread(buf, 1, sizeof buf, f)) > 0) text.append(buf, got);
    std::fclose(f);
    size_t at = text.find("\"classes\"");
    if (at == std::string::npos) return t;
    at = text.find('{', at);
    while (at != std::string::npos) {
        const size_t q0 = text.find('"', at + 1);
        const size_t close = text.find('}', at + 1);
        if (q0 == std::string::npos || (close != std::string::npos && close < q0)) break;
        const size_t q1 = text.find('"', q0 + 1);
        const size_t open = text.find('{', q1);
        const size_t end = text.find('}', open);
        if (q1 == std::string::npos || open == std::string::npos || end == std::string::npos) break;
        const int cls = std::atoi(text.substr(q0 + 1, q1 - q0 - 1).c_str());
        Tuning v = default_tuning();
        const std::string body = text.substr(open + 1, end - open - 1);
        auto knob = [&](const char* name, uint32_t* field) {
            const size_t k = body.find(std::string("\"") + name + "\"");
            if (k == std::string::npos) return;
            const size_t colon = body.find(':', k);
            if (colon != std::string::npos) *field = (uint32_t)std::atoi(body.c_str() + colon + 1);
        };
        knob("walk_blocks_per_sm", &v.walk_blocks_per_sm);
        knob("walk_max_log2", &v.walk_max_log2);
        knob("jump_block_log2", &v.jump_block_log2);
        knob("tile_max_log2", &v.tile_max_log2);
        if (cls >= 0 && cls < 64) {
            t.has[cls] = true;
            t.at[cls] = clamp_tuning(v);
        }
        at = end;
    }
    return t;
}

std::mutex g_tuning_mutex;
bool g_tuning_forced = false;
Tuning g_tuning_force{};

uint32_t size_class(uint64_t n) {
    uint32_t c = 0;
    while (c < 63 && (1ull << c) < n) ++c;
    return c;
}

Tuning tuning_for(uint64_t count) {
    static const TuningTable table = load_tuning_table();
    {
        std::lock_guard<std::mutex> lock(g_tuning_mutex);
        if (g_tuning_forced) return g_tuning_force;
    }
    const int c = (int)size_class(count);
    for (int d = 0; d < 64; ++d) {
        if (c - d >= 0 && table.has[c - d]) return table.at[c - d];
        if (c + d < 64 && table.has[c + d]) return table.at[c + d];
    }
    return default_tuning();
}

int grid_for(uint64_t work, int threads) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint64_t want = (work + threads - 1) / threads;
    const uint64_t cap = (uint64_t)sms * 16;
    return (int)std::max<uint64_t>(1, std::min<uint64_t>(want, cap));
}

// Optional per-kernel timing: when enabled, every launch is bracketed by a
// pair of events and the per-kind totals are reported after the call.
struct Recorder {
    bool enabled = false;
    std::vector<cudaEvent_t>* pool = nullptr;
    struct Mark {
        int kind;
        int level;
        size_t first; // index of the opening event
    };
    std::vector<Mark> marks;
    uint32_t launches = 0;
    int level = -1; // routing level of the launches being recorded
    cudaStream_t st = nullptr;
    size_t used = 0;

    cudaEvent_t next() {
        if (used == pool->size()) {
            cudaEvent_t e;
            check(cudaEventCreate(&e), "cudaEventCreate");
            pool->push_back(e);
        }
        return (*pool)[used++];
    }
    // `kernels`: kernel launches f makes (counted in `launches`)
    template <typename F>
    void launch(int kind, F&& f, uint32_t kernels = 1) {
        launches += kernels;
        if (!enabled) {
            f();
            return;
        }
        const size_t i = used;
        check(cudaEventRecord(next(), st), "cudaEventRecord");
        f();
        check(cudaEventRecord(next(), st), "cudaEventRecord");
        marks.push_back({kind, level, i});
    }
    void collect(double* seconds, uint32_t* counts, std::vector<Mark>* per_launch,
        std::vector<double>* per_launch_seconds) {
        per_launch->clear();
        per_launch_seconds->clear();
        for (auto& m : marks) {
            float ms = 0;
            check(cudaEventElapsedTime(&ms, (*pool)[m.first], (*pool)[m.first + 1]),
                "cudaEventElapsedTime");
            seconds[m.kind] += ms * 1e-3;
            counts[m.kind] += 1;
            per_launch->push_back(m);
            per_launch_seconds->push_back(ms * 1e-3);
        }
    }
};

// The emission launches of one section at one level, in launch order:
// f(form, full, blocks) per launch.  Packet runs of at least 32 switches
// are copied word-wise; shorter runs go out as whole words where every node
// fills the packet (transposed across 32 nodes when a cluster root holds at
// least 32 nodes, else gathered per word), and the tail packets bit by bit
// (`full` is the number of full packets, the first packet of the per-bit
// form).
// The block forms assemble words across the nodes of a cluster root, so a
// sharded level uses them only when its nodes hold whole roots.
template <typename F>
void emission_launches(const Plan& p, uint32_t l, int side, F&& f) {
    const LevelInfo& lv = p.levels[l];
    const LevelSide& ls = lv.side[side];
    const NodeRange nr = level_nodes(p, l);
    const uint32_t span_log2 = p.groups[side][ls.group].depth - ls.rel - 1;
    const uint64_t packets = (lv.cap / 2 + (1ull << span_log2) - 1) >> span_log2;
    if (span_log2 >= 5) {
        f((int)kEmitWords, 0ull, grid_for(packets << (nr.shift + span_log2 - 5), kLevelThreads));
        return;
    }
    const uint64_t half_min = lv.q / 2;
    const uint32_t rel = ls.rel;
    const uint64_t full = half_min >= 1 && nr.shift >= rel ? (half_min - 1) >> span_log2 : 0;
    const uint32_t per_word_log2 = std::min<uint32_t>(5 - span_log2, rel);
    if (full > 0 && rel >= 5) {
        const uint64_t windows = (full + (32 >> span_log2) - 1) >> (5 - span_log2);
        const uint64_t threads = (windows << (nr.shift - 5)) * 32;
        f((int)kEmitTranspose, full, grid_for(threads, kLevelThreads));
    } else if (full > 0) {
        const uint64_t words = (full << (rel - per_word_log2)) << (nr.shift - rel);
        f((int)kEmitBlocks, full, grid_for(words, kLevelThreads));
    }
    f((int)kEmitBits, full,
        grid_for((packets - std::min(packets, full)) << (nr.shift + span_log2), kLevelThreads));
}

// One global routing level: inverse (level 0 only; every later level's
// inverse comes from its parent's output pass), orbit-walk colouring
// (union-find only when the walks give up), children, then both sections'
// switch bits and the children's inverses.  `inv` holds this level's
// inverse; `child_inv` receives the next level's (null when the next level
// is the tile's, which builds its own in shared memory).
// Level 0's input still arriving from the host in parts: after wait(k) the
// stream has waited for part k, and entries [0, ends[k]) are on the device.
struct InputParts {
    std::vector<uint64_t> ends;
    std::function<void(uint32_t part)> wait;
};

template <typename TV>
void run_level(Workspace& w, Recorder& rec, cudaStream_t st, const Plan& p, const Tuning& tune,
    uint32_t l, const TV* src, uint32_t* dst, uint32_t* d_blob, uint32_t* inv,
    uint32_t* child_inv, const InputParts* input = nullptr) {
    const Plan* dp = w.d_plan;
    const LevelInfo& lv = p.levels[l];
    // the whole level's extent (array layout), and this call's share of it
    const uint64_t slots = lv.cap << l;
    const uint32_t buckets = (uint32_t)((slots + (1u << kRulerLog2) - 1) >> kRulerLog2);
    const NodeRange nr = level_nodes(p, l);
    const RulerRange rr = ruler_range(p, l);
    const uint32_t slo = (rr.lo + (1u << kSuperLog2) - 1) >> kSuperLog2;
    const uint32_t shi = (rr.hi + (1u << kSuperLog2) - 1) >> kSuperLog2;
    const uint64_t prs = lv.pcap << nr.shift;
    const uint64_t nodes = 1ull << nr.shift;
    const uint32_t my_buckets = rr.hi - rr.lo;
    const int gs = grid_for((slots + kInverseItems - 1) / kInverseItems, kLevelThreads);
    const int gu = grid_for((prs + kUnionItems - 1) / kUnionItems, kLevelThreads);
    const int gr = grid_for((prs + kResolveItems - 1) / kResolveItems, kLevelThreads);
    const int gp = grid_for(prs, kLevelThreads);
    const int gn = grid_for(nodes, kLevelThreads);
    const int gw = grid_for(my_buckets, kLevelThreads);
    uint32_t* ctl = w.control;
    // nodes whose arrays do not fit in L2 are coloured by union-find
    // 0: walks where they pay; 1: union-find everywhere; 2: walks, then the
    // union-find fallback as if they had given up (test hooks)
    const int colouring = g_force_union_find.load();
    const bool walks = lv.cap <= (1ull << tune.walk_max_log2) && colouring != 1;
    control_reset<<<1, 32, 0, st>>>(ctl, walks ? 0u : 1u);
    rec.launches += 1;
    if (l == 0 && lv.cap > kWalkMaxNode && w.records != nullptr) {
        const uint32_t windows = (uint32_t)((slots + (1ull << kPlaceLog2) - 1) >> kPlaceLog2);
        check(cudaMemsetAsync(w.cursor, 0, windows * 4, st), "cudaMemsetAsync(cursors)");
        auto bucket = [&](uint64_t lo, uint64_t hi) {
            const int gb = grid_for((hi - lo + kBucketItems - 1) / kBucketItems, kBucketThreads);
            level_bucket<TV><<<gb, kBucketThreads, 0, st>>>(dp, l, src, w.records, w.cursor, w.uf,
                w.d_status, lo, hi);
        };
        const uint32_t parts = input != nullptr ? (uint32_t)input->ends.size() : 0;
        rec.launch(kKindPlace, [&] {
            if (parts == 0) {
                bucket(0, slots);
            } else {
                // each part is bucketed as soon as it is on the device, while
                // the later parts are still being uploaded
                uint64_t lo = 0;
                for (uint32_t k = 0; k < parts; ++k) {
                    input->wait(k);
                    const uint64_t hi = std::min<uint64_t>(input->ends[k], slots);
                    if (hi > lo) bucket(lo, hi);
                    lo = std::max(lo, hi);
                }
            }
            level_place<<<grid_for(slots, kLevelThreads), kLevelThreads, 0, st>>>(dp, l,
                w.records, w.cursor, inv, ctl + kCtlClaimPlace);
        }, parts == 0 ? 2 : parts + 1);
    } else if (l == 0) {
        if (input != nullptr) {
            for (uint32_t k = 0; k < (uint32_t)input->ends.size(); ++k) input->wait(k);
        }
        rec.launch(kKindInverse, [&] {
            level_inverse<TV><<<gs, kLevelThreads, 0, st>>>(dp, l, src, inv, w.uf, w.owner,
                ctl + kCtlClaimInverse, w.d_status);
        });
    }
    rec.launch(kKindDescriptors, [&] {
        level_descriptors<<<gn, kLevelThreads, 0, st>>>(dp, l, w.addr[0], w.addr[1]);
    });
    if (walks) {
        rec.launch(kKindWalk, [&] {
            // persistent warps claiming ruler chunks in address order
            int dev = 0, sms = 148;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            const uint64_t want = ((uint64_t)my_buckets + kWalkChunk - 1) / kWalkChunk * 32;
            const int gwalk = (int)std::max<uint64_t>(1,
                std::min<uint64_t>((uint64_t)sms * tune.walk_blocks_per_sm,
                    (want + kLevelThreads - 1) / kLevelThreads));
            level_walk<TV><<<gwalk, kLevelThreads, 0, st>>>(dp, l, src, inv, w.owner,
                w.state[0], ctl);
            level_walk_short<TV><<<gp, kLevelThreads, 0, st>>>(dp, l, src, inv, w.owner, ctl);
        }, 2);
        // super-rulers of one orbit lie in one node: at most
        // (cap >> (kRulerLog2 + kSuperLog2)) + 2 of them
        const uint32_t supers = (buckets + (1u << kSuperLog2) - 1) >> kSuperLog2;
        uint32_t rounds = 1;
        while ((1ull << rounds) < (lv.cap >> (kRulerLog2 + kSuperLog2)) + 2) {
            ++rounds;
        }
        uint4* sstate[2] = {w.state[1], w.state[1] + supers};
        // few super-rulers: every round in one CTA; otherwise one launch pair per round
        const bool one_block = shi - slo <= (1u << tune.jump_block_log2);
        rec.launch(kKindJump, [&] {
            check(cudaMemsetAsync(w.super_of, 0xff, (uint64_t)buckets * 4, st),
                "cudaMemsetAsync(super rulers)");
            ruler_super_walk<<<grid_for(shi - slo, kLevelThreads), kLevelThreads, 0, st>>>(
                w.state[0], rr.lo, rr.hi, sstate[0], w.super_of, ctl);
            ruler_super_short<<<gw, kLevelThreads, 0, st>>>(w.state[0], rr.lo, rr.hi, w.super_of,
                ctl);
            if (one_block) {
                ruler_jump_block<<<1, kJumpBlockThreads, 0, st>>>(sstate[0], sstate[1], slo, shi,
                    rounds, ctl);
            } else {
                const int gj = grid_for(shi - slo, kLevelThreads);
                for (uint32_t r = 0; r <= rounds; ++r) {
                    ruler_jump<<<gj, kLevelThreads, 0, st>>>(sstate[r & 1], sstate[(r + 1) & 1],
                        slo, shi, r, ctl);
                    ruler_check<<<1, 1, 0, st>>>(r, ctl);
                }
            }
            ruler_colour<<<gw, kLevelThreads, 0, st>>>(rr.lo, rr.hi, w.super_of, sstate[0],
                sstate[1], ctl);
        }, one_block ? 4 : 3 + 2 * (rounds + 1));
        if (colouring == 2) {
            level_force_fallback<<<1, 1, 0, st>>>(ctl + kCtlHard);
            rec.launches += 1;
        }
    }
    // a walk level's union-find words are set up only if it falls back
    const bool reset_uf = walks && l > 0;
    rec.launch(kKindUnion, [&] {
        if (reset_uf) {
            level_uf_reset<<<gp, kLevelThreads, 0, st>>>(dp, l, w.uf, ctl + kCtlHard);
        }
        level_union<<<gu, kLevelThreads, 0, st>>>(dp, l, inv, w.uf, ctl + kCtlHard,
            ctl + kCtlClaimUnion, w.d_status);
    }, reset_uf ? 2 : 1);
    rec.launch(kKindOrient, [&] {
        level_orient<<<gn, kLevelThreads, 0, st>>>(dp, l, inv, w.uf, ctl + kCtlHard, w.d_status);
    });
    rec.launch(kKindResolve, [&] {
        const uint32_t supers = (buckets + (1u << kSuperLog2) - 1) >> kSuperLog2;
        level_finalize<TV><<<gr, kLevelThreads, 0, st>>>(dp, l, src, w.owner, w.super_of,
            w.state[1], w.state[1] + supers, w.uf, w.xbits, dst, ctl, w.d_status);
    });
    rec.launch(kKindOutputBits, [&] {
        // the next level's walk owners start unset and its pair-nodes as
        // roots; the tile level keeps its own state in shared memory
        const bool global_child = child_inv != nullptr;
        // owners only matter where the orbit walks run
        const bool child_walks = global_child && p.levels[l + 1].cap <= (1ull << tune.walk_max_log2)
            && colouring != 1;
        // union-find roots only for children coloured by union-find; a walk
        // child sets them up itself if it falls back (level_uf_reset)
        level_outputs<<<gp, kLevelThreads, 0, st>>>(dp, l, inv, w.xbits, w.ybits, child_inv,
            child_walks ? w.owner : nullptr, global_child && !child_walks ? w.uf : nullptr);
    });
    // above the shard level every shard computes the level, shard 0 alone
    // writes its switches
    const bool emit = p.shards <= 1 || l >= p.shard_level || p.shard == 0;
    for (int side = 0; side < 2 && emit; ++side) {
        const uint32_t* bits = side == 0 ? w.xbits : w.ybits;
        emission_launches(p, l, side, [&](int form, uint64_t full, int blocks) {
            rec.launch(kKindEmit, [&] {
                switch (form) {
                case kEmitWords:
                    level_emit_words<<<blocks, kLevelThreads, 0, st>>>(dp, l, side, bits,
                        w.addr[side], d_blob);
                    break;
                case kEmitTranspose:
                    level_emit_transpose<<<blocks, kLevelThreads, 0, st>>>(dp, l, side, bits,
                        w.addr[side], d_blob, full);
                    break;
                case kEmitBlocks:
                    level_emit_blocks<<<blocks, kLevelThreads, 0, st>>>(dp, l, side, bits,
                        w.addr[side], d_blob, full);
                    break;
                default:
                    level_emit<<<blocks, kLevelThreads, 0, st>>>(dp, l, side, bits, w.addr[side],
                        d_blob, full);
                    break;
                }
            });
        });
    }
    check(cudaGetLastError(), "level kernel launch");
}

// Raises a tile kernel's dynamic shared memory limit to the whole tile
// budget, once per kernel and device.  Setting it per call to the call's own
// size raced between concurrent callers: the limit is per function, and a
// caller that lowered it between another caller's set and launch made that
// launch fail ("too many resources requested").  The limit only bounds what
// a launch may ask for; occupancy follows each launch's actual request.
void allow_tile_smem(const void* kernel) {
    static std::mutex m;
    static std::vector<std::pair<const void*, int>> done;
    int dev = 0;
    check(cudaGetDevice(&dev), "cudaGetDevice");
    std::lock_guard<std::mutex> lock(m);
    for (const auto& d : done) {
        if (d.first == kernel && d.second == dev) return;
    }
    check(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
              (int)kTileSmemBudget),
        "cudaFuncSetAttribute");
    done.emplace_back(kernel, dev);
}

// Called after the launches of each global level are enqueued.
using LevelHook = std::function<void(uint32_t level)>;

// The tile launch split into parts at ascending tile indices (`cuts`, the
// last one the tile count), with a hook after each part's launch.
struct TileParts {
    std::vector<uint64_t> cuts;
    std::function<void(uint32_t part)> after_part;
};

template <typename T>
void launch_levels(Workspace& w, Recorder& rec, cudaStream_t st, const Plan& p,
    const TileShape& shape, const Tuning& tune, const T* d_in, uint32_t* d_blob,
    const LevelHook* after_level = nullptr, const TileParts* parts = nullptr,
    const InputParts* input = nullptr) {
    const Plan* dp = w.d_plan;
    const uint32_t t0 = p.tile_level;
    if (t0 > 0) {
        // level 0 validation: inverse slots start as 0xffffffff so a
        // duplicated value leaves a never-written slot behind
        check(cudaMemsetAsync(w.inv, 0xff, p.levels[0].cap * 4, st), "cudaMemsetAsync");
    }
    const uint32_t* cur32 = nullptr;
    uint32_t* invs[2] = {w.inv, w.inv2};
    for (uint32_t l = 0; l < t0; ++l) {
        rec.level = (int)l;
        uint32_t* dst = w.vals[l & 1];
        uint32_t* child_inv = l + 1 < t0 ? invs[(l + 1) & 1] : nullptr;
        if (l == 0) {
            run_level<T>(w, rec, st, p, tune, l, d_in, dst, d_blob, invs[0], child_inv, input);
        } else {
            run_level<uint32_t>(w, rec, st, p, tune, l, cur32, dst, d_blob, invs[l & 1],
                child_inv);
        }
        cur32 = dst;
        if (after_level != nullptr) {
            (*after_level)(l);
        }
    }
    if (t0 == 0 && input != nullptr) {
        // the tile reads the input directly: all of it first
        for (uint32_t k = 0; k < (uint32_t)input->ends.size(); ++k) input->wait(k);
    }
    rec.level = (int)t0;
    const uint64_t tiles = 1ull << level_nodes(p, t0).shift;
    if (tiles > 0x7fffffffull) {
        throw CudaFail{cudaErrorInvalidValue, "too many tiles"};
    }
    const bool wide = shape.smem > kTileSmemTwoPerSm;
    auto launch_tile = [&](auto kernel, const auto* src, unsigned threads) {
        allow_tile_smem((const void*)kernel);
        uint64_t lo = 0;
        const size_t count = parts != nullptr ? parts->cuts.size() : 1;
        for (size_t k = 0; k < count; ++k) {
            const uint64_t hi = parts != nullptr ? parts->cuts[k] : tiles;
            if (hi > lo) {
                rec.launch(kKindTile, [&] {
                    kernel<<<(unsigned)(hi - lo), threads, shape.smem, st>>>(dp, src, d_blob,
                        w.d_status, shape.slots, shape.pairs, (uint32_t)lo);
                });
            }
            if (parts != nullptr && parts->after_part) {
                parts->after_part((uint32_t)k);
            }
            lo = hi;
        }
    };
    if (t0 == 0) {
        if (wide) {
            launch_tile(tile_encode_wide<T>, d_in, 2 * kTileThreads);
        } else {
            launch_tile(tile_encode<T>, d_in, kTileThreads);
        }
    } else {
        if (wide) {
            launch_tile(tile_encode_wide<uint32_t>, cur32, 2 * kTileThreads);
        } else {
            launch_tile(tile_encode<uint32_t>, cur32, kTileThreads);
        }
    }
    check(cudaGetLastError(), "tile kernel launch");
}

struct Call {
    Layout layout;
    Plan* plan = nullptr;
    TileShape shape{};
    Tuning tune{};
};

void set_error(char* err, size_t len, const std::string& msg) {
    if (err != nullptr && len > 0) {
        std::snprintf(err, len, "%s", msg.c_str());
    }
}

Format to_format(const bpb200_format* f) {
    Format out;
    if (f == nullptr) {
        return out;
    }
    out.middle_group_log2 = f->middle_group_log2;
    out.middle_placement = f->middle_placement;
    out.input_cluster_count = f->input_cluster_count;
    out.output_cluster_count = f->output_cluster_count;
    std::memcpy(out.input_clusters, f->input_clusters, 64);
    std::memcpy(out.output_clusters, f->output_clusters, 64);
    return out;
}

// Device buffers must be aligned to the width the kernels access them with
// (4-byte blob words, entry-width input values); a misaligned pointer would
// fault on the device, so it is rejected here.
int check_device_buffers(const void* d_entries, uint32_t entry_bytes, const void* d_blob,
    char* err, size_t err_len) {
    if (((uintptr_t)d_blob & 3u) != 0) {
        set_error(err, err_len, "device blob must be 4-byte aligned");
        return kInvalidArgument;
    }
    if ((entry_bytes == 4 || entry_bytes == 8) &&
        ((uintptr_t)d_entries & (uintptr_t)(entry_bytes - 1)) != 0) {
        set_error(err, err_len, "device input must be aligned to its entry width");
        return kInvalidArgument;
    }
    return kOk;
}

// Validation shared by both entry points; fills the layout and plan.
// `tune` (null: the table's setting for `count`) fixes the tile size.
int prepare(uint64_t count, uint32_t entry_bytes, const bpb200_format* format,
    uint64_t blob_len, Workspace& w, Call* call, char* err, size_t err_len,
    const Tuning* tune = nullptr) {
    if (entry_bytes != 4 && entry_bytes != 8) {
        set_error(err, err_len, "entry width must be 4 or 8 bytes");
        return kInvalidArgument;
    }
    if (count == 0) {
        set_error(err, err_len, "permutation size is out of range");
        return kInvalidArgument;
    }
    if (entry_bytes == 4 && count > 0xffffffffull) {
        set_error(err, err_len, "permutation size requires 64-bit source values");
        return kInvalidArgument;
    }
    Error e = make_layout(count, to_format(format), &call->layout);
    if (!e.ok()) {
        set_error(err, err_len, e.message);
        return e.code;
    }
    if (count > (1ull << 31)) {
        set_error(err, err_len, "the b200 backend handles at most 2^31 entries");
        return kLength;
    }
    if (blob_len != call->layout.end_offset) {
        set_error(err, err_len, "blob length does not match the encoded size");
        return kLength;
    }
    call->plan = w.h_plan;
    call->tune = tune != nullptr ? *tune : tuning_for(count);
    const uint64_t tile_max = 1ull << call->tune.tile_max_log2;
    e = make_plan(call->layout, tile_max, call->plan);
    if (!e.ok()) {
        set_error(err, err_len, e.message);
        return e.code;
    }
    choose_tile(*call->plan, &call->shape, tile_max);
    if (call->shape.smem > kTileSmemBudget) {
        set_error(err, err_len, "tile does not fit in shared memory");
        return kLength;
    }
    return kOk;
}

// Per-thread record of the last call (the reference keeps device seconds
// thread_local too, src/benes.cpp:24).
thread_local double t_kernel_seconds[kKernelKinds];
thread_local uint32_t t_kernel_counts[kKernelKinds];
thread_local uint32_t t_launches = 0;
thread_local std::vector<Recorder::Mark> t_marks;
thread_local std::vector<double> t_mark_seconds;
std::atomic<int> g_profiling{0};

// Queues the whole encode on `st` and waits for it.
int run(Workspace& w, Call& call, cudaStream_t st, const void* d_in, uint32_t entry_bytes,
    uint32_t* d_blob, double* device_seconds, char* err, size_t err_len,
    const LevelHook* after_level = nullptr, const TileParts* parts = nullptr,
    const InputParts* input = nullptr) {
    const Plan& p = *call.plan;
    ensure_scratch(w, p);
    Recorder rec;
    rec.enabled = g_profiling.load() != 0;
    rec.pool = &w.events;
    rec.st = st;
    check(cudaMemcpyAsync(w.d_plan, w.h_plan, sizeof(Plan), cudaMemcpyHostToDevice, st),
        "plan upload");
    Header h{};
    // of the shards of one permutation only shard 0 writes the header
    h.bytes = p.shards > 1 && p.shard != 0 ? 0u : (uint32_t)call.layout.header_bytes;
    write_header(call.layout, h.data);
    check(cudaEventRecord(w.start, st), "cudaEventRecord");
    check(cudaMemsetAsync(d_blob, 0, (p.end_offset + 3) / 4 * 4, st), "cudaMemsetAsync(blob)");
    rec.launch(kKindPrologue, [&] { prologue<<<1, 128, 0, st>>>(w.d_status, d_blob, h); });
    if (entry_bytes == 4) {
        launch_levels<uint32_t>(w, rec, st, p, call.shape, call.tune, (const uint32_t*)d_in,
            d_blob, after_level, parts, input);
    } else {
        launch_levels<uint64_t>(w, rec, st, p, call.shape, call.tune, (const uint64_t*)d_in,
            d_blob, after_level, parts, input);
    }
    check(cudaEventRecord(w.stop, st), "cudaEventRecord");
    check(cudaMemcpyAsync(w.h_status, w.d_status, 4, cudaMemcpyDeviceToHost, st), "status");
    check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
    float ms = 0;
    check(cudaEventElapsedTime(&ms, w.start, w.stop), "cudaEventElapsedTime");
    if (device_seconds) {
        *device_seconds = ms * 1e-3;
    }
    for (int k = 0; k < kKernelKinds; ++k) {
        t_kernel_seconds[k] = 0;
        t_kernel_counts[k] = 0;
    }
    rec.collect(t_kernel_seconds, t_kernel_counts, &t_marks, &t_mark_seconds);
    t_launches = rec.launches;
    const uint32_t status = *w.h_status;
    if (status & kErrNotPermutation) {
        set_error(err, err_len, "input must contain every value from zero through size minus one");
        return kInvalidArgument;
    }
    if (status & (kErrIterationCap | kErrInconsistent)) {
        set_error(err, err_len, "b200 device status reported a failed colouring");
        return kRuntime;
    }
    return kOk;
}

// Whether the current device is an sm_100 part, cached per device: the
// check runs on every call, and a full cudaGetDeviceProperties costs
// milliseconds.
int current_device_ok(int* device) {
    static std::atomic<int> known[64]; // 0 unknown, 1 usable, 2 not usable
    if (cudaGetDevice(device) != cudaSuccess || *device < 0) {
        return 0;
    }
    if (*device < 64) {
        const int k = known[*device].load();
        if (k != 0) return k == 1 ? 1 : 0;
    }
    int major = 0;
    if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, *device) != cudaSuccess) {
        return 0;
    }
    const int ok = major == 10 ? 1 : 0;
    if (*device < 64) known[*device].store(ok ? 1 : 2);
    return ok;
}

template <typename Fn>
int guarded(char* err, size_t err_len, Fn&& fn) {
    try {
        return fn();
    } catch (const CudaFail& f) {
        set_error(err, err_len, std::string(f.what) + ": " + cudaGetErrorString(f.err));
        return kRuntime;
    } catch (const std::bad_alloc&) {
        set_error(err, err_len, "host allocation failed");
        return kRuntime;
    }
}

// Device staging of the host-path input and blob (grow-only).
void ensure_staging(Workspace& w, uint64_t in_bytes, uint64_t blob_len) {
    // grows at least twofold, like ensure_scratch
    if (in_bytes > w.input_cap) {
        const uint64_t cap = std::max(in_bytes, 2 * w.input_cap);
        if (w.input) cudaFree(w.input);
        w.input = nullptr;
        w.input_cap = 0;
        check(cudaMalloc(&w.input, cap), "cudaMalloc(input)");
        w.input_cap = cap;
    }
    const uint64_t blob_bytes = ((blob_len + 3) / 4 + 1) * 4;
    if (blob_bytes > w.blob_cap) {
        const uint64_t cap = std::max(blob_bytes, 2 * w.blob_cap);
        if (w.blob) cudaFree(w.blob);
        w.blob = nullptr;
        w.blob_cap = 0;
        check(cudaMalloc(&w.blob, cap), "cudaMalloc(blob)");
        w.blob_cap = cap;
    }
}

} // namespace
} // namespace bpb200

// Pinned staging rings for host copies and files.
#include "staging.inc"

namespace bpb200 {
namespace {

// Pieces of the blob that are final before the last launch, so the host
// path downloads them while the remaining work runs.  A section lists, per
// cluster group in order, each cluster's packets followed by the sections of
// its child clusters (cluster_base), so:
//  - after the last level of the first groups (the header and, per section,
//    the level-0 cluster's packets: `level`, `first[]`), when both sections
//    have more groups and those levels are all global;
//  - when the last group of both sections starts at or above the tile level,
//    after each of kTileParts tile launches: every byte before the first
//    last-group cluster whose tiles have not run yet (`cuts`, `upto[k][]`).
// The byte holding a piece's last bit may be shared with the next piece, so
// pieces end at the byte below it.
constexpr uint32_t kTileParts = 8;

struct EarlyPlan {
    bool levels = false;
    uint32_t level = 0;
    uint64_t first[2] = {0, 0};          // end of the first-group piece, per section
    std::vector<uint64_t> cuts;          // tile part ends (empty: one launch)
    std::vector<std::array<uint64_t, 2>> upto; // per part, per section: bytes final after it
};

EarlyPlan early_plan(const Plan& p) {
    EarlyPlan e;
    if (p.shards > 1 || p.tile_level == 0) {
        return e;
    }
    uint32_t last = 0;
    bool multi = true;
    for (int side = 0; side < 2; ++side) {
        if (p.group_count[side] < 2) {
            multi = false;
            break;
        }
        const GroupInfo& g = p.groups[side][0];
        last = std::max(last, g.start + g.depth - 1);
    }
    if (multi && last + 1 < p.tile_level) {
        // the single node of level 0 is small (r_0 = 0): its packets take
        // group_bits[0]
        e.levels = true;
        e.level = last;
        e.first[0] = p.section_offset[0] + p.groups[0][0].group_bits[0] / 8;
        e.first[1] = p.section_offset[1] + p.groups[1][0].group_bits[0] / 8;
    }
    uint32_t s_min = p.tile_level;
    uint32_t glast[2], slast[2];
    for (int side = 0; side < 2; ++side) {
        glast[side] = p.group_count[side] - 1;
        slast[side] = p.groups[side][glast[side]].start;
        s_min = std::min(s_min, slast[side]);
    }
    if (slast[0] > p.tile_level || slast[1] > p.tile_level || s_min == 0) {
        return e;
    }
    const uint64_t tiles = 1ull << p.tile_level;
    const uint64_t span = 1ull << (p.tile_level - s_min); // tiles per coarsest root
    if (tiles < (uint64_t)kTileParts * span || tiles < (uint64_t)kTileParts * 2048) {
        return e;
    }
    const uint64_t step = tiles / kTileParts / span * span;
    for (uint32_t k = 0; k + 1 < kTileParts; ++k) {
        const uint64_t cut = step * (k + 1);
        std::array<uint64_t, 2> at{};
        for (int side = 0; side < 2; ++side) {
            const uint64_t root = cut >> (p.tile_level - slast[side]);
            at[side] = p.section_offset[side] +
                cluster_base(p, side, glast[side], slast[side], root) / 8;
        }
        e.cuts.push_back(cut);
        e.upto.push_back(at);
    }
    e.cuts.push_back(tiles);
    return e;
}

// out[i] = (uint32_t)in[i] for i < n; true when some value needs more than
// 32 bits.  With AVX2 the stores bypass the cache (the pinned chunk is read
// next by the copy engine, not by this thread), which saves the read for
// ownership of every destination line.
__attribute__((target("avx2"))) bool narrow_values_avx2(const uint64_t* in, uint32_t* out,
    uint64_t n) {
    uint64_t i = 0;
    __m256i high = _mm256_setzero_si256();
    const __m256i pick = _mm256_setr_epi32(0, 2, 4, 6, 1, 3, 5, 7);
    if (((uintptr_t)out & 31) == 0) {
        for (; i + 8 <= n; i += 8) {
            const __m256i a = _mm256_loadu_si256(reinterpret_cast<const __m256i*>(in + i));
            const __m256i b = _mm256_loadu_si256(reinterpret_cast<const __m256i*>(in + i + 4));
            high = _mm256_or_si256(high, _mm256_or_si256(a, b));
            // low halves of a's four values, then of b's
            const __m256i la = _mm256_permutevar8x32_epi32(a, pick);
            const __m256i lb = _mm256_permutevar8x32_epi32(b, pick);
            _mm256_stream_si256(reinterpret_cast<__m256i*>(out + i),
                _mm256_permute2x128_si256(la, lb, 0x20));
        }
        _mm_sfence();
    }
    alignas(32) uint64_t lanes[4];
    _mm256_store_si256(reinterpret_cast<__m256i*>(lanes), high);
    uint64_t wide = lanes[0] | lanes[1] | lanes[2] | lanes[3];
    for (; i < n; ++i) {
        wide |= in[i];
        out[i] = (uint32_t)in[i];
    }
    return (wide >> 32) != 0;
}

bool narrow_values(const uint64_t* in, uint32_t* out, uint64_t n) {
    static const bool avx2 = __builtin_cpu_supports("avx2") != 0;
    if (avx2) {
        return narrow_values_avx2(in, out, n);
    }
    uint64_t wide = 0;
    for (uint64_t i = 0; i < n; ++i) {
        wide |= in[i];
        out[i] = (uint32_t)in[i];
    }
    return (wide >> 32) != 0;
}

constexpr uint32_t kInputParts = 8; // host-path upload parts (see compress_host)

// Narrowing of 64-bit host inputs before the upload (on unless the
// environment sets BPB200_NARROW_UPLOAD=0), with up to 16 host threads.
bool narrow_upload_enabled() {
    static const bool on = [] {
        const char* v = std::getenv("BPB200_NARROW_UPLOAD");
        return v == nullptr || std::strcmp(v, "0") != 0;
    }();
    return on;
}

int narrow_threads() {
    const unsigned hw = std::thread::hardware_concurrency();
    return (int)std::max(1u, std::min(16u, hw));
}

// Host-memory compress (bpb200_compress): upload, encode, download.
int compress_host(const void* entries, uint64_t count, uint32_t entry_bytes,
    const bpb200_format* format, uint8_t* blob, uint64_t blob_len, double* device_seconds,
    char* err, size_t err_len) {
    int device = 0;
    if (!current_device_ok(&device)) {
        set_error(err, err_len, "b200 backend is unavailable");
        return kUnavailable;
    }
    Lease lease(device);
    Workspace& w = *lease.w;
    Call call;
    int rc = prepare(count, entry_bytes, format, blob_len, w, &call, err, err_len);
    if (rc != kOk) {
        return rc;
    }
    const uint64_t in_bytes = count * entry_bytes;
    ensure_staging(w, in_bytes, blob_len);
    // 64-bit inputs of up to 2^32 entries cross PCIe as 32-bit values: the
    // ring's threads narrow them while the copy engine moves the chunks
    // already done, halving the bytes on the link.  Every valid value is
    // below count <= 2^32; a wider one means the input is not a permutation.
    const bool narrow = entry_bytes == 8 && count <= (1ull << 32) && in_bytes >= kStageMin &&
        narrow_upload_enabled();
    // Other pageable buffers of a few MB and more go through the pinned ring
    // (parallel host copies overlapping the transfer); pinned ones and small
    // ones are copied directly.
    const bool stage_in = !narrow && in_bytes >= kStageMin && !host_is_pinned(entries);
    const bool stage_out = blob_len >= kStageMin && !host_is_pinned(blob);
    std::unique_ptr<RingLease> ring;
    if (narrow || stage_in || stage_out) {
        ring = std::make_unique<RingLease>(device);
    }
    const uint32_t device_width = narrow ? 4u : entry_bytes;
    const uint64_t dev_bytes = count * device_width;
    // Narrowing fill: true when some value needs more than 32 bits.
    std::atomic<uint64_t> wide{0};
    const uint64_t* src64 = static_cast<const uint64_t*>(entries);
    const unsigned char* src8 = static_cast<const unsigned char*>(entries);
    auto fill = [&](unsigned char* dst, uint64_t len, uint64_t off) {
        if (narrow) {
            if (narrow_values(src64 + off / 4, reinterpret_cast<uint32_t*>(dst), len / 4)) {
                wide.fetch_or(1);
            }
        } else {
            std::memcpy(dst, src8 + off, len);
        }
        return true;
    };
    // When level 0 takes the partitioned inverse, the upload runs on the copy
    // stream in kInputParts parts and level 0 buckets each part as soon as it
    // is on the device (the bucket pass streams the input in order), so the
    // transfer overlaps that pass.  Part ends fall on staging-chunk bounds.
    const Plan& plan = *call.plan;
    const bool overlap = plan.shards <= 1 && plan.tile_level > 0 &&
        plan.levels[0].cap > kWalkMaxNode && dev_bytes >= kInputParts * kStageChunk;
    InputParts input;
    std::vector<uint64_t> part_bytes;
    std::mutex um;
    std::condition_variable ucv;
    uint32_t recorded = 0;
    bool upload_failed = false;
    std::thread uploader;
    struct JoinUpload {
        std::thread& t;
        ~JoinUpload() {
            if (t.joinable()) t.join();
        }
    } join_upload{uploader};
    if (overlap) {
        for (uint32_t k = 0; k < kInputParts; ++k) {
            const uint64_t want = dev_bytes / kInputParts * (k + 1);
            const uint64_t at = k + 1 == kInputParts ? dev_bytes
                : std::min(dev_bytes, (want + kStageChunk - 1) / kStageChunk * kStageChunk);
            part_bytes.push_back(at);
            input.ends.push_back(at / device_width);
        }
        if (narrow || stage_in) {
            uploader = std::thread([&] {
                uint32_t next = 0;
                const std::function<void(uint64_t)> on_issue = [&](uint64_t bytes) {
                    while (next < kInputParts && bytes >= part_bytes[next]) {
                        check(cudaEventRecord(w.inparts[next], w.copy_stream), "cudaEventRecord");
                        {
                            std::lock_guard<std::mutex> lock(um);
                            recorded = ++next;
                        }
                        ucv.notify_all();
                    }
                };
                bool ok = false;
                try {
                    ok = upload_staged(fill, dev_bytes, (unsigned char*)w.input, *ring->r,
                        w.copy_stream, narrow ? narrow_threads() : 0, &on_issue);
                } catch (const CudaFail&) {
                    ok = false;
                }
                if (!ok || next < kInputParts) {
                    std::lock_guard<std::mutex> lock(um);
                    upload_failed = true;
                }
                ucv.notify_all();
            });
            input.wait = [&](uint32_t k) {
                {
                    std::unique_lock<std::mutex> lock(um);
                    ucv.wait(lock, [&] { return upload_failed || recorded > k; });
                    if (recorded <= k) {
                        throw CudaFail{cudaErrorUnknown, "input upload"};
                    }
                }
                check(cudaStreamWaitEvent(w.stream, w.inparts[k], 0), "cudaStreamWaitEvent");
                if (k + 1 == kInputParts && uploader.joinable()) {
                    uploader.join(); // every chunk is queued; the ring is free for downloads
                }
            };
        } else {
            uint64_t lo = 0;
            for (uint32_t k = 0; k < kInputParts; ++k) {
                check(cudaMemcpyAsync((unsigned char*)w.input + lo, src8 + lo, part_bytes[k] - lo,
                          cudaMemcpyHostToDevice, w.copy_stream),
                    "input upload");
                check(cudaEventRecord(w.inparts[k], w.copy_stream), "cudaEventRecord");
                lo = part_bytes[k];
            }
            input.wait = [&](uint32_t k) {
                check(cudaStreamWaitEvent(w.stream, w.inparts[k], 0), "cudaStreamWaitEvent");
            };
        }
    } else if (narrow || stage_in) {
        upload_staged(fill, dev_bytes, (unsigned char*)w.input, *ring->r, w.stream,
            narrow ? narrow_threads() : 0);
    } else {
        check(cudaMemcpyAsync(w.input, entries, in_bytes, cudaMemcpyHostToDevice, w.stream),
            "input upload");
    }
    if (!overlap && wide.load() != 0) {
        check(cudaStreamSynchronize(w.stream), "cudaStreamSynchronize");
        set_error(err, err_len, "input must contain every value from zero through size minus one");
        return kInvalidArgument;
    }
    // Bytes [0, end) of the blob are the encoding; the first cluster groups
    // go down on the copy stream (through the ring on a helper thread for a
    // pageable blob) as soon as their last level is done.
    const uint64_t end = std::min<uint64_t>(blob_len, call.plan->end_offset);
    const unsigned char* d_bytes = (const unsigned char*)w.blob;
    auto download = [&](uint64_t off, uint64_t len, cudaStream_t st) {
        if (len == 0) {
            return;
        }
        if (stage_out) {
            if (!download_staged(
                    [blob, off](const unsigned char* src, uint64_t n, uint64_t o) {
                        std::memcpy(blob + off + o, src, n);
                        return true;
                    },
                    len, d_bytes + off, *ring->r, st)) {
                throw CudaFail{cudaErrorUnknown, "staged blob download"};
            }
        } else {
            check(cudaMemcpyAsync(blob + off, d_bytes + off, len, cudaMemcpyDeviceToHost, st),
                "blob download");
        }
    };
    // Early pieces go down on the copy stream after the event that makes
    // them final; a pageable blob goes through the ring on a helper thread,
    // which takes the pieces in order from a queue.
    EarlyPlan early;
    if (end == call.plan->end_offset) {
        early = early_plan(*call.plan);
    }
    uint64_t done[2] = {0, call.plan->section_offset[1]}; // bytes handed out, per section
    struct Piece {
        cudaEvent_t ev;
        uint64_t off, len;
    };
    std::mutex qm;
    std::condition_variable qcv;
    std::vector<Piece> queue;
    bool closed = false;
    std::atomic<int> helper_failed{0};
    std::thread helper;
    struct Join {
        std::thread& t;
        std::mutex& m;
        std::condition_variable& cv;
        bool& closed;
        ~Join() {
            {
                std::lock_guard<std::mutex> lock(m);
                closed = true;
            }
            cv.notify_all();
            if (t.joinable()) t.join();
        }
    } join{helper, qm, qcv, closed};
    if (stage_out && (early.levels || !early.cuts.empty())) {
        helper = std::thread([&] {
            size_t next = 0;
            for (;;) {
                Piece piece{};
                {
                    std::unique_lock<std::mutex> lock(qm);
                    qcv.wait(lock, [&] { return closed || next < queue.size(); });
                    if (next >= queue.size()) return;
                    piece = queue[next++];
                }
                try {
                    check(cudaStreamWaitEvent(w.copy_stream, piece.ev, 0), "cudaStreamWaitEvent");
                    download(piece.off, piece.len, w.copy_stream);
                } catch (const CudaFail&) {
                    helper_failed.store(1);
                    return;
                }
            }
        });
    }
    auto hand_out = [&](cudaEvent_t ev, const uint64_t (&to)[2]) {
        check(cudaEventRecord(ev, w.stream), "cudaEventRecord");
        for (int side = 0; side < 2; ++side) {
            const uint64_t off = side == 0 ? done[0] : done[1];
            if (to[side] <= off) continue;
            if (stage_out) {
                std::lock_guard<std::mutex> lock(qm);
                queue.push_back(Piece{ev, off, to[side] - off});
            } else {
                check(cudaStreamWaitEvent(w.copy_stream, ev, 0), "cudaStreamWaitEvent");
                download(off, to[side] - off, w.copy_stream);
            }
            done[side] = to[side];
        }
        qcv.notify_all();
    };
    const LevelHook level_hook = [&](uint32_t level) {
        if (level == early.level) {
            hand_out(w.early, early.first);
        }
    };
    TileParts parts;
    parts.cuts = early.cuts;
    parts.after_part = [&](uint32_t k) {
        if (k < early.upto.size()) {
            const uint64_t to[2] = {early.upto[k][0], early.upto[k][1]};
            hand_out(w.parts[k], to);
        }
    };
    rc = run(w, call, w.stream, w.input, device_width, w.blob, device_seconds, err, err_len,
        early.levels ? &level_hook : nullptr, early.cuts.empty() ? nullptr : &parts,
        overlap ? &input : nullptr);
    if (uploader.joinable()) {
        uploader.join();
    }
    {
        std::lock_guard<std::mutex> lock(qm);
        closed = true;
    }
    qcv.notify_all();
    if (helper.joinable()) {
        helper.join();
    }
    check(cudaStreamSynchronize(w.copy_stream), "cudaStreamSynchronize");
    if (wide.load() != 0) {
        set_error(err, err_len, "input must contain every value from zero through size minus one");
        return kInvalidArgument;
    }
    if (rc != kOk) {
        return rc;
    }
    if (helper_failed.load()) {
        throw CudaFail{cudaErrorUnknown, "staged blob download"};
    }
    // the rest: the tail of each section and whatever follows the output
    // section (the separate middle section)
    download(done[0], call.plan->section_offset[1] - done[0], w.stream);
    download(done[1], end - done[1], w.stream);
    check(cudaStreamSynchronize(w.stream), "cudaStreamSynchronize");
    return kOk;
}

} // namespace
} // namespace bpb200

using namespace bpb200;

extern "C" {

int bpb200_available(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        return 0;
    }
    int device = 0;
    return current_device_ok(&device);
}

const char* bpb200_backend_name(void) { return "b200"; }

int bpb200_encoded_size(uint64_t count, const bpb200_format* format, uint64_t* blob_bytes,
    char* err, size_t err_len) {
    Layout L;
    const Error e = make_layout(count, to_format(format), &L);
    if (!e.ok()) {
        set_error(err, err_len, e.message);
        return e.code;
    }
    *blob_bytes = L.end_offset;
    return kOk;
}

int bpb200_compress(const void* entries, uint64_t count, uint32_t entry_bytes,
    const bpb200_format* format, uint8_t* blob, uint64_t blob_len, double* device_seconds,
    char* err, size_t err_len) {
    return guarded(err, err_len, [&]() -> int {
        return compress_host(entries, count, entry_bytes, format, blob, blob_len,
            device_seconds, err, err_len);
    });
}

int bpb200_compress_device(const void* d_entries, uint64_t count, uint32_t entry_bytes,
    const bpb200_format* format, uint8_t* d_blob, uint64_t blob_len, void* stream,
    double* device_seconds, char* err, size_t err_len) {
    return guarded(err, err_len, [&]() -> int {
        int device = 0;
        if (!current_device_ok(&device)) {
            set_error(err, err_len, "b200 backend is unavailable");
            return kUnavailable;
        }
        if (const int bad = check_device_buffers(d_entries, entry_bytes, d_blob, err, err_len)) {
            return bad;
        }
        Lease lease(device);
        Workspace& w = *lease.w;
        Call call;
        int rc = prepare(count, entry_bytes, format, blob_len, w, &call, err, err_len);
        if (rc != kOk) {
            return rc;
        }
        // the work is queued on the caller's stream, after its earlier work
        return run(w, call, (cudaStream_t)stream, d_entries, entry_bytes, (uint32_t*)d_blob,
            device_seconds, err, err_len);
    });
}

int bpb200_compress_device_shard(const void* d_entries, uint64_t count, uint32_t entry_bytes,
    const bpb200_format* format, uint8_t* d_blob, uint64_t blob_len, uint32_t shard,
    uint32_t shards, void* stream, double* device_seconds, char* err, size_t err_len) {
    return guarded(err, err_len, [&]() -> int {
        int device = 0;
        if (!current_device_ok(&device)) {
            set_error(err, err_len, "b200 backend is unavailable");
            return kUnavailable;
        }
        if (shards == 0 || (shards & (shards - 1)) != 0 || shard >= shards) {
            set_error(err, err_len, "shards must be a power of two and shard below it");
            return kInvalidArgument;
        }
        if (const int bad = check_device_buffers(d_entries, entry_bytes, d_blob, err, err_len)) {
            return bad;
        }
        Lease lease(device);
        Workspace& w = *lease.w;
        Call call;
        int rc = prepare(count, entry_bytes, format, blob_len, w, &call, err, err_len);
        if (rc != kOk) {
            return rc;
        }
        uint32_t k = 0;
        while ((1u << k) < shards) ++k;
        if (k > call.plan->tile_level) {
            set_error(err, err_len, "permutation too small for that many shards");
            return kInvalidArgument;
        }
        call.plan->shards = shards;
        call.plan->shard = shard;
        call.plan->shard_level = k;
        return run(w, call, (cudaStream_t)stream, d_entries, entry_bytes, (uint32_t*)d_blob,
            device_seconds, err, err_len);
    });
}

void bpb200_set_profiling(int enabled) { g_profiling.store(enabled ? 1 : 0); }

int bpb200_get_tuning(uint64_t count, bpb200_tuning* out) {
    if (out == nullptr) return kInvalidArgument;
    const Tuning t = tuning_for(count);
    out->walk_blocks_per_sm = t.walk_blocks_per_sm;
    out->walk_max_log2 = t.walk_max_log2;
    out->jump_block_log2 = t.jump_block_log2;
    out->tile_max_log2 = t.tile_max_log2;
    return kOk;
}

int bpb200_set_tuning(const bpb200_tuning* forced) {
    std::lock_guard<std::mutex> lock(g_tuning_mutex);
    g_tuning_forced = forced != nullptr;
    if (forced != nullptr) {
        g_tuning_force = clamp_tuning(Tuning{forced->walk_blocks_per_sm, forced->walk_max_log2,
            forced->jump_block_log2, forced->tile_max_log2});
    }
    return kOk;
}

void bpb200_set_colouring(int union_find_only) {
    g_force_union_find.store(union_find_only == 2 ? 2 : (union_find_only ? 1 : 0));
}

int bpb200_describe(uint64_t count, const bpb200_format* format, uint32_t* depth,
    uint32_t* tile_level) {
    Layout L;
    const Error e = make_layout(count, to_format(format), &L);
    if (!e.ok()) {
        return e.code;
    }
    std::unique_ptr<Plan> p(new Plan);
    const uint64_t tile_max = 1ull << tuning_for(count).tile_max_log2;
    if (!make_plan(L, tile_max, p.get()).ok()) {
        return kLength;
    }
    TileShape shape;
    choose_tile(*p, &shape, tile_max);
    if (depth) *depth = p->depth;
    if (tile_level) *tile_level = p->tile_level;
    return kOk;
}

int bpb200_last_profile_launches(int* kinds, int* levels, double* seconds, int capacity) {
    const int n = (int)t_marks.size();
    for (int i = 0; i < n && i < capacity; ++i) {
        if (kinds) kinds[i] = t_marks[i].kind;
        if (levels) levels[i] = t_marks[i].level;
        if (seconds) seconds[i] = t_mark_seconds[i];
    }
    return n;
}

int bpb200_last_profile(double* seconds, uint32_t* launches, int kinds, uint32_t* total_launches) {
    const int n = kinds < kKernelKinds ? kinds : kKernelKinds;
    for (int k = 0; k < n; ++k) {
        if (seconds) seconds[k] = t_kernel_seconds[k];
        if (launches) launches[k] = t_kernel_counts[k];
    }
    if (total_launches) *total_launches = t_launches;
    return kKernelKinds;
}

void bpb200_shutdown(void) {
    std::lock_guard<std::mutex> lock(g_pool_mutex);
    for (auto& w : g_pool) {
        if (!w->busy) {
            w->destroy();
        }
    }
    g_pool.erase(std::remove_if(g_pool.begin(), g_pool.end(),
                     [](const std::unique_ptr<Workspace>& w) { return w->device < 0; }),
        g_pool.end());
    destroy_rings();
}

int bpb200_probe_switch_bit(uint64_t count, const bpb200_format* format, int side,
    uint32_t level, uint64_t node, uint64_t pair, uint64_t* bit) {
    Layout L;
    if (!make_layout(count, to_format(format), &L).ok()) {
        return kInvalidArgument;
    }
    std::unique_ptr<Plan> p(new Plan);
    if (!make_plan(L, kTileMaxEntries, p.get()).ok()) {
        return kInvalidArgument;
    }
    if (level >= L.depth || node >= (1ull << level) || (side != 0 && side != 1)) {
        return kInvalidArgument;
    }
    const uint64_t size = node_size(p->levels[level], level, node);
    if (size <= p->leaf || pair >= size / 2) {
        return kInvalidArgument;
    }
    *bit = switch_bit(node_address(*p, side, level, node), pair);
    return kOk;
}

int bpb200_probe_rank_bit(uint64_t count, const bpb200_format* format, uint32_t level,
    uint64_t node, int* section, uint64_t* bit) {
    Layout L;
    if (!make_layout(count, to_format(format), &L).ok()) {
        return kInvalidArgument;
    }
    std::unique_ptr<Plan> p(new Plan);
    if (!make_plan(L, kTileMaxEntries, p.get()).ok()) {
        return kInvalidArgument;
    }
    if (level > L.depth || node >= (1ull << level)) {
        return kInvalidArgument;
    }
    if (node_size(p->levels[level], level, node) > p->leaf) {
        return kInvalidArgument;
    }
    *bit = leaf_rank_bit(*p, level, node, section);
    return kOk;
}

} // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free entry point.
//
// Some callers cannot call cudaMalloc: processes whose device memory is
// owned by a pooling allocator that must account for every byte, and
// latency-critical paths that cannot afford the device-wide synchronisation
// cudaMalloc/cudaFree can imply.  For them,
// bpb200_compress_device_noalloc runs the same encode with all of its
// scratch (plan, status word, level arrays, inverse, union-find words,
// colour bits, node descriptors) carved out of one file-scope device array
// of fixed size.  The array exists on every GPU that loads this library and
// stays allocated until the process exits.
// ---------------------------------------------------------------------------
namespace bpb200 {
namespace noalloc {

constexpr uint64_t kMaxEntries = 1ull << 18;          // largest permutation accepted
constexpr uint64_t kSlots = kMaxEntries + (1ull << 14); // level slots incl. padding
constexpr uint64_t kPairs = kSlots / 2 + (1ull << 13);
constexpr uint64_t kNodes = 1ull << 10;               // descriptors per global level

constexpr size_t up256(size_t x) { return (x + 255) / 256 * 256; }
constexpr size_t kOffPlan = 0;
constexpr size_t kOffStatus = kOffPlan + up256(sizeof(Plan));
constexpr size_t kOffVals0 = kOffStatus + 256;
constexpr size_t kOffVals1 = kOffVals0 + up256(kSlots * 4);
constexpr size_t kOffInv = kOffVals1 + up256(kSlots * 4);
constexpr size_t kOffInv2 = kOffInv + up256(kSlots * 4);
constexpr size_t kOffUf = kOffInv2 + up256(kSlots * 4);
constexpr size_t kOffXbits = kOffUf + up256(kPairs * 4);
constexpr size_t kOffYbits = kOffXbits + up256((kPairs / 32 + 1) * 4);
constexpr size_t kOffAddr0 = kOffYbits + up256((kPairs / 32 + 1) * 4);
constexpr size_t kOffAddr1 = kOffAddr0 + up256(kNodes * sizeof(NodeAddress));
constexpr size_t kOffOwner = kOffAddr1 + up256(kNodes * sizeof(NodeAddress));
constexpr size_t kOffState0 = kOffOwner + up256(kPairs * 4);
constexpr size_t kOffState1 = kOffState0 + up256(((kSlots >> kRulerLog2) + 1) * sizeof(uint4));
constexpr size_t kOffSuper = kOffState1 + up256(((kSlots >> kRulerLog2) + 1) * sizeof(uint4));
constexpr size_t kOffControl = kOffSuper + up256(((kSlots >> kRulerLog2) + 1) * 4);
constexpr size_t kBytes = kOffControl + 256; // under 8 MB
static_assert(kBytes < (8u << 20), "allocation-free scratch stays under 8 MB");

} // namespace noalloc
} // namespace bpb200

// The scratch itself.  In host code this name is only a host-side stand-in,
// not a device address; the device address is obtained per device with
// cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char bpb200_noalloc_scratch[bpb200::noalloc::kBytes];

namespace bpb200 {
namespace noalloc {

constexpr int kMaxDevices = 64;
std::mutex g_mutex;                    // guards the two tables below
unsigned char* g_scratch[kMaxDevices]; // device address of the array, per device
Plan g_plan;                           // host staging of the plan (no heap, no pinning)

} // namespace noalloc
} // namespace bpb200

extern "C" int bpb200_compress_device_noalloc(const void* d_entries, uint64_t count,
    uint32_t entry_bytes, const bpb200_format* format, uint8_t* d_blob, uint64_t blob_len,
    void* stream, char* err, size_t err_len) {
    using namespace bpb200;
    return guarded(err, err_len, [&]() -> int {
        int device = 0;
        if (!current_device_ok(&device)) {
            set_error(err, err_len, "b200 backend is unavailable");
            return kUnavailable;
        }
        if (device < 0 || device >= noalloc::kMaxDevices) {
            set_error(err, err_len, "device ordinal out of range for the allocation-free entry point");
            return kRuntime;
        }
        if (count > noalloc::kMaxEntries) {
            set_error(err, err_len,
                "the allocation-free entry point accepts at most 262144 (2^18) entries");
            return kLength;
        }
        if (const int bad = check_device_buffers(d_entries, entry_bytes, d_blob, err, err_len)) {
            return bad;
        }
        // One host thread at a time stages the plan; device-side overlap of
        // two calls is the caller's to avoid (they would share the scratch).
        std::lock_guard<std::mutex> lock(noalloc::g_mutex);
        if (noalloc::g_scratch[device] == nullptr) {
            // first call on this device: resolve the array's device address
            // (callers make this first call before capturing any stream)
            void* ptr = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&ptr, bpb200_noalloc_scratch);
            if (e != cudaSuccess || ptr == nullptr) {
                set_error(err, err_len, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
                return kRuntime;
            }
            noalloc::g_scratch[device] = static_cast<unsigned char*>(ptr);
        }
        unsigned char* base = noalloc::g_scratch[device];
        Workspace w; // views into the static array; owns nothing
        w.h_plan = &noalloc::g_plan;
        Call call;
        const Tuning fixed = default_tuning(); // the scratch limits assume the compiled tile size
        int rc = prepare(count, entry_bytes, format, blob_len, w, &call, err, err_len, &fixed);
        if (rc != kOk) {
            return rc;
        }
        const Plan& p = *call.plan;
        const uint64_t nodes = p.tile_level > 0 ? (1ull << (p.tile_level - 1)) : 0;
        if ((p.tile_level > 0 && (p.max_slots > noalloc::kSlots || p.max_pairs > noalloc::kPairs)) ||
            nodes > noalloc::kNodes) {
            set_error(err, err_len, "format needs more scratch than the allocation-free entry point holds");
            return kLength;
        }
        w.d_plan = reinterpret_cast<Plan*>(base + noalloc::kOffPlan);
        w.d_status = reinterpret_cast<uint32_t*>(base + noalloc::kOffStatus);
        w.vals[0] = reinterpret_cast<uint32_t*>(base + noalloc::kOffVals0);
        w.vals[1] = reinterpret_cast<uint32_t*>(base + noalloc::kOffVals1);
        w.inv = reinterpret_cast<uint32_t*>(base + noalloc::kOffInv);
        w.inv2 = reinterpret_cast<uint32_t*>(base + noalloc::kOffInv2);
        w.uf = reinterpret_cast<uint32_t*>(base + noalloc::kOffUf);
        w.xbits = reinterpret_cast<uint32_t*>(base + noalloc::kOffXbits);
        w.ybits = reinterpret_cast<uint32_t*>(base + noalloc::kOffYbits);
        w.addr[0] = reinterpret_cast<NodeAddress*>(base + noalloc::kOffAddr0);
        w.addr[1] = reinterpret_cast<NodeAddress*>(base + noalloc::kOffAddr1);
        w.owner = reinterpret_cast<uint32_t*>(base + noalloc::kOffOwner);
        w.state[0] = reinterpret_cast<uint4*>(base + noalloc::kOffState0);
        w.state[1] = reinterpret_cast<uint4*>(base + noalloc::kOffState1);
        w.super_of = reinterpret_cast<uint32_t*>(base + noalloc::kOffSuper);
        w.control = reinterpret_cast<uint32_t*>(base + noalloc::kOffControl);
        cudaStream_t st = (cudaStream_t)stream;
        // The plan source is ordinary host memory: the copy is staged before
        // cudaMemcpyAsync returns, so g_plan can be reused by the next call.
        check(cudaMemcpyAsync(w.d_plan, &noalloc::g_plan, sizeof(Plan), cudaMemcpyHostToDevice, st),
            "plan upload");
        Header h{};
        h.bytes = (uint32_t)call.layout.header_bytes;
        write_header(call.layout, h.data);
        // Everything that must start cleared is cleared by the call itself:
        // the blob (memset), the status word (prologue) and, when level
        // kernels run, the inverse sentinels used for validation.
        check(cudaMemsetAsync(d_blob, 0, (p.end_offset + 3) / 4 * 4, st), "cudaMemsetAsync(blob)");
        Recorder rec; // timing disabled: no events are created
        rec.st = st;
        rec.launch(kKindPrologue, [&] { prologue<<<1, 128, 0, st>>>(w.d_status, (uint32_t*)d_blob, h); });
        if (entry_bytes == 4) {
            launch_levels<uint32_t>(w, rec, st, p, call.shape, call.tune, (const uint32_t*)d_entries,
                (uint32_t*)d_blob);
        } else {
            launch_levels<uint64_t>(w, rec, st, p, call.shape, call.tune, (const uint64_t*)d_entries,
                (uint32_t*)d_blob);
        }
        uint32_t status = 0;
        check(cudaMemcpyAsync(&status, w.d_status, 4, cudaMemcpyDeviceToHost, st), "status");
        check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
        if (status & kErrNotPermutation) {
            set_error(err, err_len, "input must contain every value from zero through size minus one");
            return kInvalidArgument;
        }
        if (status & (kErrIterationCap | kErrInconsistent)) {
            set_error(err, err_len, "b200 device status reported a failed colouring");
            return kRuntime;
        }
        return kOk;
    });
}

// Batched and serving forms (share this file's pool, planning and launches).
#include "serve.inc"

// File form: streamed file -> device -> file (compress_file).
#include "file.inc"

// Batch lookup verifier (device twin of the reference's lookup).
#include "lookup.inc"

// Random-access roofline probe.
#include "probe.inc"
