// Device runtime behind the C ABI: per-context device memory, the tick's
// launch sequence, host-pointer mirrors, status checks with capacity regrow,
// the learned closure's per-tick steps and training driver, the device tick
// loop, and the batched ensemble's CUDA graphs.
//
// Ownership follows the reference (polesitter.h:1699-1767): the caller owns
// every particle array and the ps_config_t buffer, and the host-side state
// lives inside that buffer.  The device scratch (sorted particles, tree,
// near lists) is cudaMalloc'ed in ps_init from max_particles and freed in
// ps_destroy; it replaces the reference's arena + radix temporaries.
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <cmath>
#include <mutex>
#include <new>
#include <vector>

#include "psg_closure.cuh"
#include "psg_common.cuh"
#include "psg_kernels.h"

namespace psg {

static thread_local char g_err[256];

static void note(const char* what, cudaError_t e) {
    std::snprintf(g_err, sizeof(g_err), "%s: %s", what, cudaGetErrorString(e));
}

#define PSG_CHECK(call)                        \
    do {                                       \
        cudaError_t _e = (call);               \
        if (_e != cudaSuccess) {               \
            ::psg::note(#call, _e);            \
            return PSG_EDEVICE;                \
        }                                      \
    } while (0)

#define PSG_ALLOC(ptr, bytes)                                        \
    do {                                                             \
        cudaError_t _e = cudaMalloc((void**)&(ptr), (bytes) ? (bytes) : 16); \
        if (_e != cudaSuccess) {                                     \
            ::psg::note("cudaMalloc " #ptr, _e);                     \
            return PSG_EALLOC;                                       \
        }                                                            \
    } while (0)

constexpr uint32_t kMagic = 0x50534732u;  // "PSG2"
constexpr int kPhases = 9;  // timing events
enum Phase { PH_SORT = 0, PH_GATHER, PH_TREE, PH_UP, PH_TRAV, PH_END, PH_BEGIN, PH_CLOSURE,
             PH_DENSE };

struct Mirror {
    float *x, *y, *z, *m, *fx, *fy, *fz;
    uint32_t *id, *codes;
    size_t cap;
};

// the learned closure's device buffers (allocated when it is first enabled)
struct ClosureState {
    int mode;            // 0 off (the reference), 1 order-1 local, 2 order-1 + MLP
    int judge;           // run the sampled FP64 judge in mode 1 too
    int judge_bps;       // blocks per SM of the judge's FP64 direct sum (1..8)
    int judge_samples;   // particles of the judge's sample (64..kJudgeSamples)
    float4* lg0;         // per node: field gradient xx yy zz xy
    float2* lg1;         //           xz yz
    uint32_t* leaf_of;   // per sorted particle: its leaf
    float4* dF;          // per sorted particle: the MLP's correction
    float* params;       // FP32 parameter vector (kMlpParams)
    MlpPacked* packed;   // BF16 device copy
    int have_weights;
    uint32_t* judge_tg;  // judge sample (sorted indices)
    double* judge_f64;   // FP64 direct forces of the sample
    double* judge_part;  // ... their partial sums per source split
    size_t judge_part_n;
    JudgeOut* d_judge;
    JudgeOut* h_judge;
    uint32_t tick;       // ticks run in closure mode (varies the judge sample)
    JudgeOut last;       // judge result of the last tick (samples 0: none)
    int valid;           // the last completed tick ran the order-1 traversal
    cudaStream_t side;   // the judge's direct sum, beside the tree and traversal
    cudaEvent_t ev_sorted, ev_judge;
};

struct State {
    uint32_t magic;
    int device;
    int sms;
    int trav_grid[2][2][2];  // leaf-pass grid [closure order 0 / 1][sparse / dense variant]
                             // [plain / chain + stream variant]
    int trav_int_grid[2];
    size_t max_particles;
    float theta;
    int morton_variant;
    int debug;
    int timing;
    cudaStream_t stream;
    float4* xyzm;
    uint32_t* ids;
    SortBuffers sort;
    uint32_t* tree_tiles;
    TreeView tv;
    uint32_t* ns;
    unsigned long long ns_cap;
    P2PStore p2p;
    uint4* dense_rec;      // full-leaf P2P work records
    uint32_t dense_cap;
    uint2* dense_part;     // per warp of k_dense_p2p: its record's partial entries
    uint32_t dense_part_warps;
    uint32_t* heavy_frontier;
    uint32_t heavy_fcap;
    int heavy_slots;       // blocks of k_heavy_leaf
    cudaStream_t aux;      // k_heavy_leaf, beside the leaf pass
    cudaEvent_t ev_levels, ev_heavy;
    // host-array calls: the sorted arrays (final after the gather) go back to
    // pinned host buffers on their own stream while the traversal runs
    struct EarlyCopy {
        void* h;
        const void* dv;
    } early[6];
    int n_early = 0;
    size_t early_bytes = 0;
    bool early_issued = false;
    cudaStream_t copy_out = nullptr;
    cudaEvent_t ev_written = nullptr, ev_copied = nullptr;
    int heavy_depth;       // option; < 0: derived from theta
    int forest_heavy;      // many systems: the deepest of their shallow-leaf depths
    int ns_levels;         // near lists are stored for node depths <= this (kMaxDepth: all);
                           // lowered when they do not fit, deeper groups walk their chains
    int stream_p2p;        // P2P summed in the leaf pass as found (no spill store)
    int force_ns_levels;   // option: store near lists for depths <= this at most
    int force_stream;      // option: always stream the P2P
    int sort_spin_limit;   // look-back polls before the sort gives up (option; 0: default)
    uint32_t leaf_cap;     // option: nodes holding more particles are split (1: the reference)
    double grid_scale;     // traversal grids x this (ensemble autotuner); 0: 1
    int kahan;
    Status* d_status;
    Status* h_status;
    Mirror mir;
    cudaEvent_t ev[kPhases];
    float ms[kPhases];
    unsigned long long stats[24];
    uint32_t last_nodes;
    uint32_t lvl_count[kLevels];  // node counts of the last completed tick
    // device tick loop scratch (allocated by its first call)
    int tk_grid;
    float2* tk_partial;
    float* tk_bbox;
    float* tk_v[3];
    float* tk_vmir[3];
    ClosureState cl;
    int order;  // traversal's local expansion order: 0 (reference) or 1
    size_t last_n;  // particles of the last completed tick
    size_t trav_n;  // particles of the tick whose traversal is being enqueued
    int attempts;   // traversal runs of the last tick (> 1: a capacity regrow)
};

// the near-list levels and the P2P mode start over when what they depend
// on (theta, leaf capacity, expansion order, store sizes) changes
static void reset_near_levels(State* s) {
    s->ns_levels = kMaxDepth;
    s->stream_p2p = 0;
}

static int grid_for(const State* s, size_t n, int per_block_items) {
    size_t want = (n + per_block_items - 1) / per_block_items;
    size_t cap = (size_t)s->sms * 8;
    if (want < 1) want = 1;
    return (int)(want < cap ? want : cap);
}

static int alloc_ns(State* s, unsigned long long cap) {
    if (s->ns) cudaFree(s->ns);
    s->ns = nullptr;
    s->ns_cap = 0;
    PSG_ALLOC(s->ns, cap * sizeof(uint32_t));
    s->ns_cap = cap;
    return PSG_OK;
}

static int alloc_p2p(State* s, uint32_t chunks) {
    void* ps[4] = {s->p2p.src, s->p2p.mask, s->p2p.next, s->p2p.cnt};
    for (void* p : ps)
        if (p) cudaFree(p);
    s->p2p.src = s->p2p.next = s->p2p.cnt = nullptr;
    s->p2p.mask = nullptr;
    s->p2p.cap_chunks = 0;
    PSG_ALLOC(s->p2p.src, (size_t)chunks * kP2PChunk * 4);
    PSG_ALLOC(s->p2p.mask, (size_t)chunks * kP2PChunk);
    PSG_ALLOC(s->p2p.next, (size_t)chunks * 4);
    PSG_ALLOC(s->p2p.cnt, (size_t)chunks * 4);
    s->p2p.cap_chunks = chunks;
    return PSG_OK;
}

static int alloc_dense(State* s, uint32_t cap) {
    if (s->dense_rec) cudaFree(s->dense_rec);
    s->dense_rec = nullptr;
    s->dense_cap = 0;
    PSG_ALLOC(s->dense_rec, (size_t)cap * sizeof(uint4));
    s->dense_cap = cap;
    return PSG_OK;
}

// blocks of k_dense_p2p for n particles: the blocks that fit on the SMs,
// fewer for a small system (whose records, if any, are few), so an ensemble
// of small systems does not launch thousands of idle blocks each
static size_t dense_grid(const State* s, size_t n) {
    return std::min<size_t>((size_t)s->sms * kDenseBlocksPerSm, std::max<size_t>(4, n / 64));
}

// frontier buffers of k_heavy_leaf: 2 x cap candidates per block
static int alloc_heavy(State* s, uint32_t cap) {
    if (s->heavy_frontier) cudaFree(s->heavy_frontier);
    s->heavy_frontier = nullptr;
    // per block: two frontiers and the P2P source list of a multi-particle leaf
    PSG_ALLOC(s->heavy_frontier, (size_t)s->heavy_slots * 3 * cap * 4);
    s->heavy_fcap = cap;
    return PSG_OK;
}

static int ensure_mirror(Mirror& mi, size_t n) {
    if (mi.cap >= n) return PSG_OK;
    void** ps[9] = {(void**)&mi.x, (void**)&mi.y, (void**)&mi.z, (void**)&mi.m, (void**)&mi.fx,
                    (void**)&mi.fy, (void**)&mi.fz, (void**)&mi.id, (void**)&mi.codes};
    for (auto p : ps) {
        if (*p) cudaFree(*p);
        *p = nullptr;
    }
    for (auto p : ps) {
        cudaError_t e = cudaMalloc(p, n * 4 ? n * 4 : 16);
        if (e != cudaSuccess) {
            note("cudaMalloc mirror", e);
            return PSG_EALLOC;
        }
    }
    mi.cap = n;
    return PSG_OK;
}

static void free_mirror(Mirror& mi) {
    void* ps[9] = {mi.x, mi.y, mi.z, mi.m, mi.fx, mi.fy, mi.fz, mi.id, mi.codes};
    for (auto p : ps)
        if (p) cudaFree(p);
    std::memset(&mi, 0, sizeof(mi));
}

// true when the GPU can dereference p (device or managed memory)
static bool pinned_host(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

static bool on_device(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

static void free_state(State* s) {
    void* ps[] = {s->xyzm, s->ids, s->sort.key_a, s->sort.key_b, s->sort.val_a, s->sort.val_b,
                  s->sort.hist, s->sort.offs, s->sort.lookback, s->tree_tiles, s->tv.geo,
                  s->tv.mp, s->tv.lt, s->tv.info, s->tv.parent, s->tv.arrive, s->tv.cbase,
                  s->tv.ns_off, s->tv.ns_cnt, s->tv.dbg_m2l, s->tv.dbg_p2p, s->tv.link,
                  s->tv.p2p_head, s->ns, s->p2p.src, s->p2p.mask, s->p2p.next, s->p2p.cnt,
                  s->d_status, s->dense_rec, s->dense_part, s->heavy_frontier, s->tk_partial, s->tk_bbox, s->tk_v[0], s->tk_v[1], s->tk_v[2],
                  s->tk_vmir[0], s->tk_vmir[1], s->tk_vmir[2], s->cl.lg0, s->cl.lg1,
                  s->cl.leaf_of, s->cl.dF, s->cl.params, s->cl.packed, s->cl.judge_tg,
                  s->cl.judge_f64, s->cl.judge_part, s->cl.d_judge};
    for (void* p : ps)
        if (p) cudaFree(p);
    if (s->h_status) cudaFreeHost(s->h_status);
    if (s->cl.h_judge) cudaFreeHost(s->cl.h_judge);
    if (s->cl.side) cudaStreamSynchronize(s->cl.side);
    if (s->cl.ev_sorted) cudaEventDestroy(s->cl.ev_sorted);
    if (s->cl.ev_judge) cudaEventDestroy(s->cl.ev_judge);
    if (s->cl.side) cudaStreamDestroy(s->cl.side);
    free_mirror(s->mir);
    for (int i = 0; i < kPhases; ++i)
        if (s->ev[i]) cudaEventDestroy(s->ev[i]);
    if (s->aux) {
        cudaStreamSynchronize(s->aux);
        cudaStreamDestroy(s->aux);
    }
    if (s->ev_levels) cudaEventDestroy(s->ev_levels);
    if (s->ev_heavy) cudaEventDestroy(s->ev_heavy);
    if (s->copy_out) {
        cudaStreamSynchronize(s->copy_out);
        cudaStreamDestroy(s->copy_out);
    }
    if (s->ev_written) cudaEventDestroy(s->ev_written);
    if (s->ev_copied) cudaEventDestroy(s->ev_copied);
    if (s->stream) cudaStreamDestroy(s->stream);
    s->magic = 0;
}

// lvl_caps (optional): node capacity of each level, for a tree pass over
// many systems; sort_passes: radix passes the look-back flags must serve
static int init_state(State* s, size_t maxp, float theta, const uint32_t* lvl_caps = nullptr,
                      int sort_passes = 4) {
    std::memset(s, 0, sizeof(State));
    PSG_CHECK(cudaGetDevice(&s->device));
    PSG_CHECK(cudaDeviceGetAttribute(&s->sms, cudaDevAttrMultiProcessorCount, s->device));
    PSG_CHECK(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    for (int i = 0; i < kPhases; ++i) PSG_CHECK(cudaEventCreate(&s->ev[i]));
    s->max_particles = maxp;
    s->theta = theta;
    s->morton_variant = PSG_MORTON_AVX2;
    const size_t n = maxp ? maxp : 1;
    PSG_ALLOC(s->xyzm, n * sizeof(float4));
    PSG_ALLOC(s->ids, n * 4);
    PSG_ALLOC(s->sort.key_a, n * 4);
    PSG_ALLOC(s->sort.key_b, n * 4);
    PSG_ALLOC(s->sort.val_a, n * 4);
    PSG_ALLOC(s->sort.val_b, n * 4);
    PSG_ALLOC(s->sort.hist, 4 * 256 * 4);
    PSG_ALLOC(s->sort.offs, 4 * 256 * 4);
    const size_t stiles = (n + sort_tile_size() - 1) / sort_tile_size();
    PSG_ALLOC(s->sort.lookback, (size_t)sort_passes * stiles * 256 * 4);
    const size_t ttiles = (n + tree_tile_size() - 1) / tree_tile_size();
    PSG_ALLOC(s->tree_tiles, ttiles * kMaxDepth * 4);
    // level capacities: min(8^d, n) nodes at depth d
    uint32_t base = 0;
    for (int d = 0; d <= kMaxDepth; ++d) {
        unsigned long long cap8 = 1ull << (3 * d);
        uint32_t cap = (uint32_t)(cap8 < n ? cap8 : n);
        if (d == 0) cap = 1;
        if (lvl_caps) cap = lvl_caps[d];
        s->tv.lvl_base[d] = base;
        s->tv.lvl_cap[d] = cap;
        base += cap;
    }
    s->tv.lvl_base[kLevels] = base;
    s->tv.lvl_cap[kLevels] = 0;
    const size_t nodes = base;
    PSG_ALLOC(s->tv.geo, nodes * 16);
    PSG_ALLOC(s->tv.mp, nodes * 16);
    PSG_ALLOC(s->tv.lt, nodes * 16);
    PSG_ALLOC(s->tv.info, nodes * 16);
    PSG_ALLOC(s->tv.parent, nodes * 4);
    PSG_ALLOC(s->tv.arrive, nodes * 4);
    PSG_ALLOC(s->tv.cbase, nodes * 4);
    PSG_ALLOC(s->tv.ns_off, nodes * 4);
    PSG_ALLOC(s->tv.ns_cnt, nodes * 4);
    PSG_ALLOC(s->tv.dbg_m2l, nodes * 4);
    PSG_ALLOC(s->tv.dbg_p2p, nodes * 4);
    PSG_ALLOC(s->tv.link, nodes * 4);
    PSG_ALLOC(s->tv.p2p_head, nodes * 4);
    PSG_ALLOC(s->d_status, sizeof(Status));
    PSG_CHECK(cudaMallocHost((void**)&s->h_status, sizeof(Status)));
    std::memset(s->h_status, 0, sizeof(Status));
    int r = alloc_ns(s, (unsigned long long)(n < 1024 ? 1024 : n) * 48ull);
    if (r != PSG_OK) return r;
    r = alloc_p2p(s, (uint32_t)(n < 4096 ? 4096 : n / 4));
    if (r != PSG_OK) return r;
    r = alloc_dense(s, (uint32_t)(n / 4 + 1024));
    if (r != PSG_OK) return r;
    s->dense_part_warps = (uint32_t)dense_grid(s, n) * kDenseWarpsPerBlock;
    PSG_ALLOC(s->dense_part, (size_t)s->dense_part_warps * kDensePartCap * sizeof(uint2));
    // shallow leaves: a frontier holds at most one level's nodes plus the
    // parent's near list
    s->heavy_slots = 64;
    r = alloc_heavy(s, (uint32_t)(n / 4 + 4096));
    if (r != PSG_OK) return r;
    s->heavy_depth = -1;
    s->ns_levels = kMaxDepth;
    s->force_ns_levels = kMaxDepth;
    s->leaf_cap = 1;
    PSG_CHECK(cudaStreamCreateWithFlags(&s->aux, cudaStreamNonBlocking));
    PSG_CHECK(cudaEventCreateWithFlags(&s->ev_levels, cudaEventDisableTiming));
    PSG_CHECK(cudaEventCreateWithFlags(&s->ev_heavy, cudaEventDisableTiming));
    for (int o = 0; o < 2; ++o) {
        int bps = 0;
        for (int dn = 0; dn < 2; ++dn) {
            for (int xl = 0; xl < 2; ++xl) {
                PSG_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                    &bps, traverse_kernel_ptr(o, dn, xl), traverse_threads(), 0));
                s->trav_grid[o][dn][xl] = s->sms * (bps > 0 ? bps : 1);
            }
        }
        PSG_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &bps, traverse_internal_kernel_ptr(o), traverse_threads(), 0));
        s->trav_int_grid[o] = s->sms * (bps > 0 ? bps : 1);
    }
    s->magic = kMagic;
    return PSG_OK;
}

static int closure_alloc(State* s) {
    ClosureState& c = s->cl;
    if (c.lg0) return PSG_OK;
    const size_t nodes = s->tv.lvl_base[kLevels];
    const size_t n = s->max_particles ? s->max_particles : 1;
    PSG_ALLOC(c.lg0, nodes * sizeof(float4));
    PSG_ALLOC(c.lg1, nodes * sizeof(float2));
    PSG_ALLOC(c.leaf_of, n * 4);
    PSG_ALLOC(c.dF, n * sizeof(float4));
    PSG_ALLOC(c.params, kMlpParams * sizeof(float));
    PSG_ALLOC(c.packed, sizeof(MlpPacked));
    PSG_ALLOC(c.judge_tg, kJudgeSamples * 4);
    PSG_ALLOC(c.judge_f64, kJudgeSamples * 3 * sizeof(double));
    c.judge_part_n = direct_f64_part_doubles(n, kJudgeSamples, s->sms * 8);
    if (c.judge_bps == 0) c.judge_bps = 4;
    if (c.judge_samples == 0) c.judge_samples = kJudgeDefault;
    PSG_ALLOC(c.judge_part, c.judge_part_n * sizeof(double));
    PSG_ALLOC(c.d_judge, sizeof(JudgeOut));
    PSG_CHECK(cudaMallocHost((void**)&c.h_judge, sizeof(JudgeOut)));
    std::memset(c.h_judge, 0, sizeof(JudgeOut));
    PSG_CHECK(cudaStreamCreateWithFlags(&c.side, cudaStreamNonBlocking));
    PSG_CHECK(cudaEventCreateWithFlags(&c.ev_sorted, cudaEventDisableTiming));
    PSG_CHECK(cudaEventCreateWithFlags(&c.ev_judge, cudaEventDisableTiming));
    return PSG_OK;
}

// Leaves at most this deep are walked block-parallel by k_heavy_leaf: a leaf
// at depth d (half width H / 2^d of the root's H) stays unseparated from the
// sources within about theta H / 2^(d-1), a large part of the tree once
// 2^d <= 4 theta.  That only costs a warp long in a large system: below
// kHeavyMinParticles, where a walk over the whole tree is still short (and
// shallow leaves are most leaves), the leaf pass takes every leaf.
constexpr size_t kHeavyMinParticles = 131072;

static int heavy_depth_of(float theta, size_t n) {
    if (n < kHeavyMinParticles) return 0;
    int d = 0;
    while (d < 5 && (float)(2 << d) <= 4.0f * theta) ++d;
    return d < 2 ? 2 : d;
}

static int heavy_depth_for(const State* s) {
    if (s->tv.part_sys) return s->forest_heavy;  // many systems: the deepest of theirs
    if (s->heavy_depth >= 0) return s->heavy_depth > 5 ? 5 : s->heavy_depth;
    return heavy_depth_of(s->theta, s->trav_n);
}

// Depth of the deepest nodes whose near lists this traversal stores.  The
// shallow-leaf walk reads the lists of depths < heavy_depth, so they always
// exist; the order-1 expansion needs every level's (its chain groups would
// need each ancestor's own gradient).
static int near_levels(const State* s) {
    if (s->order >= 1) return kMaxDepth;
    int k = std::min(s->ns_levels, s->force_ns_levels);
    return std::max(k, std::max(2, heavy_depth_for(s) - 1));
}

static void record(State* s, int ph) {
    if (s->timing) cudaEventRecord(s->ev[ph], s->stream);
}

// one traversal run (internal levels, leaf pass, shallow leaves, full
// leaves) enqueued on s->stream; no host synchronisation
static int enqueue_traversal(State* s, const float4* xyzm, float* fx, float* fy, float* fz) {
    PSG_CHECK(cudaMemsetAsync(&s->d_status->work[0], 0, sizeof(s->d_status->work), s->stream));
    PSG_CHECK(cudaMemsetAsync(&s->d_status->ns_used[0], 0, sizeof(s->d_status->ns_used),
                              s->stream));
    PSG_CHECK(cudaMemsetAsync(&s->d_status->p2p_chunks, 0, 4, s->stream));
    PSG_CHECK(cudaMemsetAsync(&s->d_status->dense_count, 0, 8, s->stream));
    PSG_CHECK(cudaMemsetAsync(&s->d_status->heavy_work, 0, 4, s->stream));
    PSG_CHECK(cudaMemsetAsync(&s->d_status->ns_fail, 0, 4, s->stream));
    TravArgs A;
    A.tv = s->tv;
    A.p2p = s->p2p;
    A.ns = s->ns;
    A.ns_cap = s->ns_cap;
    A.status = s->d_status;
    A.theta = s->theta;
    A.level = 0;
    A.debug = s->debug;
    A.kahan = s->kahan;
    A.xyzm = xyzm;
    A.fx = fx;
    A.fy = fy;
    A.fz = fz;
    const int o = s->order >= 1 ? 1 : 0;
    A.order = o;
    A.leaf_of = o ? s->cl.leaf_of : nullptr;
    A.tv.lg0 = o ? s->cl.lg0 : nullptr;
    A.tv.lg1 = o ? s->cl.lg1 : nullptr;
    A.dense_rec = s->dense_rec;
    A.dense_cap = s->dense_cap;
    A.dense_part = s->dense_part;
    A.dense_part_warps = s->dense_part_warps;
    A.heavy_depth = heavy_depth_for(s);
    A.heavy_frontier = s->heavy_frontier;
    A.heavy_fcap = s->heavy_fcap;
    A.ns_levels = near_levels(s);
    A.leaf_cap = s->leaf_cap;
    A.stream = (s->stream_p2p || s->force_stream) ? 1 : 0;
    const double gs = s->grid_scale > 0.0 ? s->grid_scale : 1.0;
    auto scaled = [&](int g) {
        const int v = (int)(g * gs);
        return v < 1 ? 1 : v;
    };
    // Shallow leaves on the aux stream.  Their walk reads the near lists and
    // fields of the groups above depth heavy_depth, final once the internal
    // level of depth heavy_depth - 1 is done, so it starts there and runs
    // beside the deeper levels and the leaf pass (which starts at the groups
    // of depth heavy_depth).
    bool heavy_started = false;
    auto start_heavy = [&]() -> int {
        PSG_CHECK(cudaEventRecord(s->ev_levels, s->stream));
        PSG_CHECK(cudaStreamWaitEvent(s->aux, s->ev_levels, 0));
        launch_heavy_leaf(A, scaled(s->heavy_slots), s->aux);
        PSG_CHECK(cudaEventRecord(s->ev_heavy, s->aux));
        heavy_started = true;
        return PSG_OK;
    };
    const int heavy_ready = A.heavy_depth - 1;
    if (heavy_ready < 2) {
        const int r = start_heavy();
        if (r != PSG_OK) return r;
    }
    for (int k = 2; k <= A.ns_levels; ++k) {
        launch_traverse_internal(A, k, scaled(s->trav_int_grid[o]), s->stream);
        if (k == heavy_ready) {
            const int r = start_heavy();
            if (r != PSG_OK) return r;
        }
    }
    record(s, PH_TRAV);
    if (!heavy_started) {
        const int r = start_heavy();
        if (r != PSG_OK) return r;
    }
    // one system: the leaf pass starts past the shallow groups; many: each
    // group checks its own system's depth
    launch_leaf_start(s->d_status, s->tv.part_sys ? 0 : A.heavy_depth, o, s->stream);
    const int xl = (A.ns_levels < kMaxDepth || A.stream) ? 1 : 0;
    const int lg[2] = {scaled(s->trav_grid[o][0][xl]), scaled(s->trav_grid[o][1][xl])};
    launch_traverse_leaves(A, lg, s->stream);
    record(s, PH_DENSE);
    launch_dense_p2p(A, scaled((int)dense_grid(s, s->trav_n)), s->stream);
    PSG_CHECK(cudaStreamWaitEvent(s->stream, s->ev_heavy, 0));
    record(s, PH_END);
    return PSG_OK;
}

// bytes a growing store may take: what the device has free plus what the
// store holds now (freed before the new one is allocated), less 1/16 of the
// device for everything else
static unsigned long long store_budget(unsigned long long held) {
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
        cudaGetLastError();
        return held;
    }
    const unsigned long long avail = (unsigned long long)fr + held, margin = tot / 16;
    return avail > margin ? avail - margin : 0ull;
}

// a store of another size, or the old one back when the device refuses
static bool try_alloc_ns(State* s, unsigned long long cap) {
    const unsigned long long old = s->ns_cap;
    if (alloc_ns(s, cap) == PSG_OK) return true;
    cudaGetLastError();
    alloc_ns(s, old);
    return false;
}

static bool try_alloc_p2p(State* s, uint32_t chunks) {
    const uint32_t old = s->p2p.cap_chunks;
    if (alloc_p2p(s, chunks) == PSG_OK) return true;
    cudaGetLastError();
    alloc_p2p(s, old);
    return false;
}

// After a traversal run read back its status, makes room for every store
// that ran out, for the rerun and later ticks:
//  * near lists: grown to twice what the run reserved while the device has
//    the memory and 32-bit offsets reach; past that (order 0), they stop at
//    the level before the first that did not fit, the groups below walk
//    their ancestor chains, and the P2P is streamed, so no store grows with
//    theta any more;
//  * P2P chunks: grown likewise, else the P2P is streamed;
//  * full-leaf records and shallow-leaf frontiers: grown.
// PSG_EOOM when nothing can give.
static int regrow(State* s, uint32_t err) {
    if (err & PSG_ERR_NS_OVERFLOW) {
        const unsigned long long used = s->h_status->ns_used[0];
        const uint32_t fail = s->h_status->ns_fail;
        const int kf = fail ? __builtin_ctz(fail) : kMaxDepth;
        const unsigned long long limit =
            std::min(0xFFFFFFF0ull, store_budget(s->ns_cap * 4) / 4);
        const unsigned long long want = 2 * used + (1ull << 20);
        const int floor_k = std::max(2, heavy_depth_for(s) - 1);
        bool done = false;
        if (want <= limit) {
            done = try_alloc_ns(s, want);
        } else if (s->ns_cap < limit && used + (1ull << 20) <= limit) {
            // what the run reserved fits, twice that does not: the largest
            // store, and the levels below show whether it is enough
            done = try_alloc_ns(s, limit);
        }
        if (!done && s->order == 0 && kf - 1 >= floor_k) {
            s->ns_levels = kf - 1;
            s->stream_p2p = 1;
            done = true;
        }
        if (!done && s->order >= 1 && limit > s->ns_cap) done = try_alloc_ns(s, limit);
        if (!done) {
            std::snprintf(g_err, sizeof(g_err),
                          "near lists need %llu entries at level %d; the device holds %llu",
                          want, kf, limit);
            return PSG_EOOM;
        }
    }
    if (err & PSG_ERR_HEAVY_OVERFLOW) {
        unsigned long long cap = 2ull * s->heavy_fcap;
        const unsigned long long most = 2ull * s->max_particles + 1024;
        int r = alloc_heavy(s, (uint32_t)(cap < most ? cap : most));
        if (r != PSG_OK) return r;
    }
    if (err & PSG_ERR_DENSE_OVERFLOW) {
        unsigned long long need = s->h_status->dense_count;
        need = need + need / 4 + 1024;
        if (need > 0x7FFFFFFFull) need = 0x7FFFFFFFull;
        int r = alloc_dense(s, (uint32_t)need);
        if (r != PSG_OK) return r;
    }
    if (err & PSG_ERR_P2P_OVERFLOW) {
        // the chunk counter is 32-bit: below the capacity it has wrapped
        const unsigned long long used = s->h_status->p2p_chunks;
        const unsigned long long need = used < s->p2p.cap_chunks ? ~0ull : 2 * used + 1024;
        const unsigned long long per = kP2PChunk * 5 + 8;
        const unsigned long long limit =
            std::min(0x7FFFFFFFull, store_budget(s->p2p.cap_chunks * per) / per);
        if (!(need <= limit && try_alloc_p2p(s, (uint32_t)need))) s->stream_p2p = 1;
    }
    return PSG_OK;
}

// traversal of all levels + P2P/L2P; regrows the near-list regions or the
// P2P chunk store and reruns when a capacity flag comes back
static int run_traversal(State* s, const float4* xyzm, float* fx, float* fy, float* fz,
                         uint32_t* err_out) {
    for (int attempt = 0; attempt < 6; ++attempt) {
        s->attempts = attempt + 1;
        int r0 = enqueue_traversal(s, xyzm, fx, fy, fz);
        if (r0 != PSG_OK) return r0;
        PSG_CHECK(cudaGetLastError());
        PSG_CHECK(cudaMemcpyAsync(s->h_status, s->d_status, sizeof(Status),
                                  cudaMemcpyDeviceToHost, s->stream));
        PSG_CHECK(cudaStreamSynchronize(s->stream));
        const uint32_t err = s->h_status->err;
        if (!(err & (PSG_ERR_NS_OVERFLOW | PSG_ERR_P2P_OVERFLOW | PSG_ERR_DENSE_OVERFLOW |
                     PSG_ERR_HEAVY_OVERFLOW))) {
            *err_out = err;
            return PSG_OK;
        }
        int rg = regrow(s, err);
        if (rg != PSG_OK) return rg;
        PSG_CHECK(cudaMemsetAsync(&s->d_status->err, 0, 4, s->stream));
        PSG_CHECK(cudaMemsetAsync(&s->d_status->stat[0], 0, sizeof(s->d_status->stat), s->stream));
        if (s->timing) cudaEventRecord(s->ev[PH_UP], s->stream);
    }
    std::snprintf(g_err, sizeof(g_err), "traversal stores still too small after 6 runs");
    return PSG_EOOM;
}

// the caller's arrays as the GPU sees them: in place when it can reach them,
// else device mirrors in the context
struct DevArrays {
    float *x, *y, *z, *m, *fx, *fy, *fz;
    uint32_t *id, *codes;
    bool dev[9];
    bool any_host;
};

static int map_arrays(State* s, const psg_arrays_t* a, DevArrays& d, bool upload_codes) {
    const size_t n = a->n;
    d.x = a->x; d.y = a->y; d.z = a->z; d.m = a->mass;
    d.fx = a->fx; d.fy = a->fy; d.fz = a->fz; d.id = a->id; d.codes = a->codes;
    void* ps[9] = {d.x, d.y, d.z, d.m, d.fx, d.fy, d.fz, d.id, d.codes};
    d.any_host = false;
    for (int i = 0; i < 9; ++i) {
        d.dev[i] = on_device(ps[i]);
        d.any_host |= !d.dev[i];
    }
    if (!d.any_host) return PSG_OK;
    int r = ensure_mirror(s->mir, s->max_particles);
    if (r != PSG_OK) return r;
    struct { void* h; void* dv; bool in; } io[9] = {
        {a->x, s->mir.x, true}, {a->y, s->mir.y, true}, {a->z, s->mir.z, true},
        {a->mass, s->mir.m, true}, {a->fx, s->mir.fx, false}, {a->fy, s->mir.fy, false},
        {a->fz, s->mir.fz, false}, {a->id, s->mir.id, true}, {a->codes, s->mir.codes, upload_codes}};
    for (int i = 0; i < 9; ++i)
        if (!d.dev[i] && io[i].in)
            PSG_CHECK(cudaMemcpyAsync(io[i].dv, io[i].h, n * 4, cudaMemcpyHostToDevice, s->stream));
    if (!d.dev[0]) d.x = s->mir.x;
    if (!d.dev[1]) d.y = s->mir.y;
    if (!d.dev[2]) d.z = s->mir.z;
    if (!d.dev[3]) d.m = s->mir.m;
    if (!d.dev[4]) d.fx = s->mir.fx;
    if (!d.dev[5]) d.fy = s->mir.fy;
    if (!d.dev[6]) d.fz = s->mir.fz;
    if (!d.dev[7]) d.id = s->mir.id;
    if (!d.dev[8]) d.codes = s->mir.codes;
    return PSG_OK;
}

static int unmap_arrays(State* s, const psg_arrays_t* a, const DevArrays& d) {
    if (!d.any_host) return PSG_OK;
    struct { void* h; void* dv; } out[9] = {
        {a->x, d.x}, {a->y, d.y}, {a->z, d.z}, {a->mass, d.m}, {a->fx, d.fx},
        {a->fy, d.fy}, {a->fz, d.fz}, {a->id, d.id}, {a->codes, d.codes}};
    for (int i = 0; i < 9; ++i)
        if (!d.dev[i])
            PSG_CHECK(cudaMemcpyAsync(out[i].h, out[i].dv, a->n * 4, cudaMemcpyDeviceToHost,
                                      s->stream));
    return PSG_OK;
}

// ps_calc_forces on device-resident arrays: sort -> gather -> tree -> upward
// -> traversal (polesitter.h:1840-1909).  The root is (cx, cy, cz, hw), or,
// when bbox is set, derived on the device from this tick's bounding box.
static int tick_core(State* s, const DevArrays& d, size_t n, float cx, float cy, float cz,
                     float hw, const float* bbox) {
    cudaStream_t st = s->stream;
    record(s, PH_BEGIN);
    PSG_CHECK(cudaMemsetAsync(s->d_status, 0, sizeof(Status), st));
    const int g = grid_for(s, n, 1024);
    launch_sort(s->sort, d.codes, n, g, s->d_status, st, s->sort_spin_limit);
    record(s, PH_SORT);
    launch_gather(s->sort.perm, d.x, d.y, d.z, d.m, d.id, n, s->xyzm, s->ids, g, st);
    launch_writeback(s->xyzm, s->ids, n, d.x, d.y, d.z, d.m, d.id, g, st);
    if (s->n_early && !s->early_issued) {
        PSG_CHECK(cudaEventRecord(s->ev_written, st));
        PSG_CHECK(cudaStreamWaitEvent(s->copy_out, s->ev_written, 0));
        for (int k = 0; k < s->n_early; ++k)
            PSG_CHECK(cudaMemcpyAsync(s->early[k].h, s->early[k].dv, s->early_bytes,
                                      cudaMemcpyDeviceToHost, s->copy_out));
        PSG_CHECK(cudaEventRecord(s->ev_copied, s->copy_out));
        s->early_issued = true;
    }
    record(s, PH_GATHER);
    // closure judge: its FP64 direct sum needs only the sorted particles, so
    // it runs on a side stream under the tree build and traversal, on a
    // quarter of the GPU's block slots
    ClosureState& cj = s->cl;
    const bool judge = s->order >= 1 && n > 1 && ((cj.mode == 2 && cj.have_weights) || cj.judge);
    const int smp = n < (size_t)cj.judge_samples ? (int)n : cj.judge_samples;
    if (judge) {
        PSG_CHECK(cudaEventRecord(cj.ev_sorted, st));
        PSG_CHECK(cudaStreamWaitEvent(cj.side, cj.ev_sorted, 0));
        launch_judge_direct(s->xyzm, n, cj.judge_tg, smp, cj.judge_f64, cj.tick,
                            s->sms * cj.judge_bps,
                            cj.side, cj.judge_part, cj.judge_part_n);
        PSG_CHECK(cudaEventRecord(cj.ev_judge, cj.side));
    }
    const int gt = (int)((s->tv.lvl_base[kLevels] + 255) / 256);
    if (s->debug) {
        PSG_CHECK(cudaMemsetAsync(s->tv.dbg_m2l, 0, (size_t)s->tv.lvl_base[kLevels] * 4, st));
        PSG_CHECK(cudaMemsetAsync(s->tv.dbg_p2p, 0, (size_t)s->tv.lvl_base[kLevels] * 4, st));
    }
    launch_tree(d.codes, n, s->tree_tiles, s->tv, s->d_status, cx, cy, cz, hw, gt, st, bbox,
                s->leaf_cap);
    record(s, PH_TREE);
    launch_upward(s->tv, s->d_status, s->xyzm, gt, st);
    record(s, PH_UP);
    PSG_CHECK(cudaGetLastError());
    uint32_t err = 0;
    if (n == 1) {
        // a single particle: the root is a leaf and its only P2P term is
        // the zero self-interaction (polesitter.h:1279-1449)
        PSG_CHECK(cudaMemsetAsync(d.fx, 0, 4, st));
        PSG_CHECK(cudaMemsetAsync(d.fy, 0, 4, st));
        PSG_CHECK(cudaMemsetAsync(d.fz, 0, 4, st));
        record(s, PH_TRAV);
        record(s, PH_DENSE);
        record(s, PH_END);
        PSG_CHECK(cudaMemcpyAsync(s->h_status, s->d_status, sizeof(Status),
                                  cudaMemcpyDeviceToHost, st));
        PSG_CHECK(cudaStreamSynchronize(st));
        err = s->h_status->err;
    } else {
        s->trav_n = n;
        int r = run_traversal(s, s->xyzm, d.fx, d.fy, d.fz, &err);
        if (r != PSG_OK) {
            if (judge) cudaStreamSynchronize(cj.side);  // leave no judge work running
            return r;
        }
    }
    if (err & (PSG_ERR_SORT_SPIN | PSG_ERR_STACK | PSG_ERR_NODES | PSG_ERR_HEAVY_OVERFLOW |
               PSG_ERR_CHAIN_ORDER)) {
        if (judge) cudaStreamSynchronize(cj.side);
        const bool nodes = (err & PSG_ERR_NODES) &&
                           !(err & (PSG_ERR_SORT_SPIN | PSG_ERR_STACK | PSG_ERR_HEAVY_OVERFLOW |
                                    PSG_ERR_CHAIN_ORDER));
        std::snprintf(g_err, sizeof(g_err), nodes ? "morton codes not sorted/30-bit (0x%x)"
                                                  : "device status error 0x%x", err);
        return nodes ? PSG_EINVAL : PSG_EDEVICE;
    }
    s->cl.last.samples = 0;
    s->cl.valid = s->order >= 1 && n > 1;
    if (judge) {
        // learned closure: MLP correction, the judge's decision, fallback
        ClosureState& c = s->cl;
        const bool mlp = c.mode == 2 && c.have_weights;
        {
            TreeView tv = s->tv;
            tv.lg0 = c.lg0;
            tv.lg1 = c.lg1;
            if (mlp) {
                launch_closure_mlp(tv, c.leaf_of, s->xyzm, n, c.packed, c.dF, s->sms,
                                   &s->d_status->err, st);
            } else {
                PSG_CHECK(cudaMemsetAsync(c.dF, 0, n * sizeof(float4), st));
            }
            PSG_CHECK(cudaStreamWaitEvent(st, c.ev_judge, 0));
            launch_judge_decide(c.judge_tg, smp, c.judge_f64, d.fx, d.fy, d.fz, c.dF,
                                mlp ? 1 : 0, c.d_judge, st);
            if (mlp) launch_closure_apply(d.fx, d.fy, d.fz, c.dF, n, c.d_judge, s->sms, st);
            PSG_CHECK(cudaGetLastError());
            PSG_CHECK(cudaMemcpyAsync(c.h_judge, c.d_judge, sizeof(JudgeOut),
                                      cudaMemcpyDeviceToHost, st));
            if (mlp)
                PSG_CHECK(cudaMemcpyAsync(&s->h_status->err, &s->d_status->err, 4,
                                          cudaMemcpyDeviceToHost, st));
            PSG_CHECK(cudaStreamSynchronize(st));
            if (mlp && (s->h_status->err & PSG_ERR_TC_TIMEOUT)) {
                std::snprintf(g_err, sizeof(g_err),
                              "closure network: a tensor-core MMA did not complete");
                return PSG_EDEVICE;
            }
            c.last = *c.h_judge;
            ++c.tick;
        }
    }
    record(s, PH_CLOSURE);
    uint32_t nodes = 0;
    for (int k = 0; k <= kMaxDepth; ++k) {
        s->lvl_count[k] = s->h_status->lvl_count[k];
        nodes += s->lvl_count[k];
    }
    s->last_nodes = nodes;
    s->last_n = n;
    for (int i = 0; i < 8; ++i) s->stats[i] = s->h_status->stat[i];
    s->stats[8] = nodes;
    s->stats[9] = s->h_status->max_stack;
    for (int i = 8; i < 16; ++i) s->stats[i + 8] = s->h_status->stat[i];
    s->stats[10] = s->h_status->p2p_chunks;
    s->stats[11] = (unsigned long long)s->attempts;
    s->stats[12] = s->h_status->max_leaf;
    s->stats[13] = s->h_status->dense_count;
    s->stats[14] = (unsigned long long)near_levels(s);
    s->stats[15] = (s->stream_p2p || s->force_stream) ? 1ull : 0ull;
    if (s->timing) {
        cudaEventSynchronize(s->ev[PH_CLOSURE]);
        const int order[7] = {PH_BEGIN, PH_SORT, PH_GATHER, PH_TREE, PH_UP, PH_TRAV, PH_DENSE};
        for (int i = 0; i + 1 < 7; ++i)
            cudaEventElapsedTime(&s->ms[i], s->ev[order[i]], s->ev[order[i + 1]]);
        cudaEventElapsedTime(&s->ms[6], s->ev[PH_BEGIN], s->ev[PH_CLOSURE]);
        cudaEventElapsedTime(&s->ms[7], s->ev[PH_END], s->ev[PH_CLOSURE]);
        cudaEventElapsedTime(&s->ms[8], s->ev[PH_DENSE], s->ev[PH_END]);
    }
    return PSG_OK;
}

static int calc(State* s, const psg_arrays_t* a, float cx, float cy, float cz, float hw) {
    const size_t n = a->n;
    if (n > s->max_particles) return PSG_EINVAL;
    if (n == 0) return PSG_OK;
    PSG_CHECK(cudaSetDevice(s->device));
    DevArrays d;
    int r = map_arrays(s, a, d, true);
    if (r != PSG_OK) return r;
    // sorted positions, masses, ids and codes into pinned host arrays go back
    // while the traversal runs (a pageable copy would block this thread, so
    // those wait for the end); the forces go back at the end
    s->n_early = 0;
    s->early_issued = false;
    s->early_bytes = n * 4;
    if (d.any_host) {
        void* const hs[6] = {a->x, a->y, a->z, a->mass, a->id, a->codes};
        const void* const ds[6] = {d.x, d.y, d.z, d.m, d.id, d.codes};
        const int which[6] = {0, 1, 2, 3, 7, 8};
        for (int k = 0; k < 6; ++k) {
            if (d.dev[which[k]] || !pinned_host(hs[k])) continue;
            s->early[s->n_early++] = State::EarlyCopy{hs[k], ds[k]};
            d.dev[which[k]] = true;  // (unmap_arrays skips it)
        }
        if (s->n_early && !s->copy_out) {
            PSG_CHECK(cudaStreamCreateWithFlags(&s->copy_out, cudaStreamNonBlocking));
            PSG_CHECK(cudaEventCreateWithFlags(&s->ev_written, cudaEventDisableTiming));
            PSG_CHECK(cudaEventCreateWithFlags(&s->ev_copied, cudaEventDisableTiming));
        }
    }
    r = tick_core(s, d, n, cx, cy, cz, hw, nullptr);
    if (r == PSG_OK) r = unmap_arrays(s, a, d);
    if (s->early_issued) {
        // the forces' copies and the tick's end wait for the early copies too
        const cudaError_t e = cudaStreamWaitEvent(s->stream, s->ev_copied, 0);
        if (e != cudaSuccess && r == PSG_OK) {
            note("cudaStreamWaitEvent", e);
            r = PSG_EDEVICE;
        }
        cudaStreamSynchronize(s->copy_out);
    }
    s->n_early = 0;
    s->early_issued = false;
    if (r != PSG_OK) return r;
    PSG_CHECK(cudaStreamSynchronize(s->stream));
    return PSG_OK;
}

// `ticks` iterations of the caller's loop (README.md:65-111) without leaving
// the device: ids reset, prepare, calc with the root derived on the device,
// velocities permuted through ids, semi-implicit Euler.  Host arrays are
// copied in once and out once.
static int run_ticks(State* s, const psg_arrays_t* a, float* vx, float* vy, float* vz, float dt,
                     uint32_t ticks, int variant) {
    const size_t n = a->n;
    if (n > s->max_particles) return PSG_EINVAL;
    if (n == 0 || ticks == 0) return PSG_OK;
    PSG_CHECK(cudaSetDevice(s->device));
    cudaStream_t st = s->stream;
    if (!s->tk_bbox) {
        s->tk_grid = s->sms * 4;
        PSG_ALLOC(s->tk_partial, s->tk_grid * sizeof(float2));
        PSG_ALLOC(s->tk_bbox, 4 * sizeof(float));
        for (int c = 0; c < 3; ++c) PSG_ALLOC(s->tk_v[c], s->max_particles * 4);
        for (int c = 0; c < 3; ++c) PSG_ALLOC(s->tk_vmir[c], s->max_particles * 4);
    }
    DevArrays d;
    int r = map_arrays(s, a, d, false);
    if (r != PSG_OK) return r;
    float* vh[3] = {vx, vy, vz};
    float* vin[3];
    float* vout[3];
    for (int c = 0; c < 3; ++c) {
        if (on_device(vh[c])) {
            vin[c] = vh[c];
        } else {
            vin[c] = s->tk_vmir[c];
            PSG_CHECK(cudaMemcpyAsync(vin[c], vh[c], n * 4, cudaMemcpyHostToDevice, st));
        }
        vout[c] = s->tk_v[c];
    }
    float* const vdst[3] = {vin[0], vin[1], vin[2]};
    const int g = grid_for(s, n, 1024);
    int gp = (int)((n + 1023) / 1024);
    if (gp > s->tk_grid) gp = s->tk_grid;
    for (uint32_t t = 0; t < ticks; ++t) {
        launch_tick_reset_ids(d.id, n, g, st);
        launch_prepare(d.x, d.y, d.z, n, s->tk_partial, gp, d.codes, s->tk_bbox, variant, st);
        r = tick_core(s, d, n, 0.f, 0.f, 0.f, 0.f, s->tk_bbox);
        if (r != PSG_OK) return r;
        TickState ts;
        ts.id = d.id;
        ts.vx_in = vin[0]; ts.vy_in = vin[1]; ts.vz_in = vin[2];
        ts.vx_out = vout[0]; ts.vy_out = vout[1]; ts.vz_out = vout[2];
        ts.x = d.x; ts.y = d.y; ts.z = d.z; ts.m = d.m;
        ts.fx = d.fx; ts.fy = d.fy; ts.fz = d.fz;
        launch_tick_euler(ts, n, dt, g, st);
        PSG_CHECK(cudaGetLastError());
        for (int c = 0; c < 3; ++c) {
            float* tmp = vin[c];
            vin[c] = vout[c];
            vout[c] = tmp;
        }
    }
    for (int c = 0; c < 3; ++c) {
        if (vin[c] != vdst[c])
            PSG_CHECK(cudaMemcpyAsync(vdst[c], vin[c], n * 4, cudaMemcpyDeviceToDevice, st));
        if (vdst[c] != vh[c])
            PSG_CHECK(cudaMemcpyAsync(vh[c], vdst[c], n * 4, cudaMemcpyDeviceToHost, st));
    }
    r = unmap_arrays(s, a, d);
    if (r != PSG_OK) return r;
    PSG_CHECK(cudaStreamSynchronize(st));
    return PSG_OK;
}

// ---- process-wide workspace of ps_prepare_particles (it takes no context) ----
struct PrepWs {
    std::mutex mu;
    int device = -1;
    cudaStream_t stream = nullptr;
    float2* partial = nullptr;
    float* bbox = nullptr;
    float* h_bbox = nullptr;
    int grid = 0;
    Mirror mir{};
};
static PrepWs g_prep;

static int prepare(const psg_arrays_t* a, float* out_min, float* out_max, float* out_range,
                   int variant) {
    std::lock_guard<std::mutex> lock(g_prep.mu);
    int dev = 0;
    PSG_CHECK(cudaGetDevice(&dev));
    if (g_prep.device != dev) {
        if (g_prep.stream) {
            cudaSetDevice(g_prep.device);
            cudaStreamDestroy(g_prep.stream);
            cudaFree(g_prep.partial);
            cudaFree(g_prep.bbox);
            cudaFreeHost(g_prep.h_bbox);
            free_mirror(g_prep.mir);
            cudaSetDevice(dev);
        }
        int sms = 0;
        PSG_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        PSG_CHECK(cudaStreamCreateWithFlags(&g_prep.stream, cudaStreamNonBlocking));
        g_prep.grid = sms * 4;
        PSG_ALLOC(g_prep.partial, g_prep.grid * sizeof(float2));
        PSG_ALLOC(g_prep.bbox, 4 * sizeof(float));
        PSG_CHECK(cudaMallocHost((void**)&g_prep.h_bbox, 4 * sizeof(float)));
        g_prep.device = dev;
    }
    const size_t n = a->n;
    cudaStream_t st = g_prep.stream;
    const float* x = a->x; const float* y = a->y; const float* z = a->z;
    uint32_t* codes = a->codes;
    const bool dx = on_device(x), dy = on_device(y), dz = on_device(z), dc = on_device(codes);
    if (!(dx && dy && dz && dc)) {
        int r = ensure_mirror(g_prep.mir, n);
        if (r != PSG_OK) return r;
        if (!dx) { PSG_CHECK(cudaMemcpyAsync(g_prep.mir.x, x, n * 4, cudaMemcpyHostToDevice, st)); x = g_prep.mir.x; }
        if (!dy) { PSG_CHECK(cudaMemcpyAsync(g_prep.mir.y, y, n * 4, cudaMemcpyHostToDevice, st)); y = g_prep.mir.y; }
        if (!dz) { PSG_CHECK(cudaMemcpyAsync(g_prep.mir.z, z, n * 4, cudaMemcpyHostToDevice, st)); z = g_prep.mir.z; }
        if (!dc) codes = g_prep.mir.codes;
    }
    int grid = (int)((n + 1023) / 1024);
    if (grid > g_prep.grid) grid = g_prep.grid;
    if (grid < 1) grid = 1;
    launch_prepare(x, y, z, n, g_prep.partial, grid, codes, g_prep.bbox, variant, st);
    PSG_CHECK(cudaGetLastError());
    if (!dc) PSG_CHECK(cudaMemcpyAsync(a->codes, codes, n * 4, cudaMemcpyDeviceToHost, st));
    PSG_CHECK(cudaMemcpyAsync(g_prep.h_bbox, g_prep.bbox, 4 * sizeof(float), cudaMemcpyDeviceToHost, st));
    PSG_CHECK(cudaStreamSynchronize(st));
    if (out_min) *out_min = g_prep.h_bbox[0];
    if (out_max) *out_max = g_prep.h_bbox[1];
    if (out_range) *out_range = g_prep.h_bbox[2];
    return PSG_OK;
}

// ---- batched ensemble: many independent systems in one tree pass ----------
//
// All systems share one set of device buffers: their particles are the
// caller's concatenated arrays (system k at [off_k, off_k + N_k)), and every
// phase of the tick is one launch over all of them -- the segmented bounding
// box and Morton codes, the radix sort (four code passes, then stable passes
// on the system index, so each system ends sorted within its range), the
// tree build (a system's first position starts its root, node k of level 0;
// no run crosses a system boundary), the level-synchronous upward pass, and
// the persistent traversal kernels, whose work queues run over the groups of
// every system with each group's own theta, root, leaf-pass variant and
// shallow-leaf depth.  Per system the arithmetic is exactly that of its own
// tick, so the results equal each system's ps_b200_run_ticks bit for bit.
// One tick is two CUDA graphs captured once and replayed (forces; velocity
// permutation + Euler); between them the host reads the one status block and
// regrows a store that ran out (then that traversal is rerun and the graphs
// are captured again).

constexpr uint32_t kEnsMagic = 0x50534745u;  // "PSGE"
constexpr uint32_t kForestBlock = 1024;      // particles per prepare block

struct Ensemble {
    uint32_t magic = 0;
    int device = 0;
    size_t nsys = 0, total = 0;
    std::vector<size_t> count, offset;
    std::vector<float> theta;       // per system
    std::vector<uint32_t> cap;      // leaf capacity per system
    State* fs = nullptr;            // the device state of all systems together
    // per-system tables (device)
    uint32_t* part_sys = nullptr;   // system of each particle position
    uint32_t* sys_off = nullptr;    // [nsys + 1]
    uint32_t* sys_cap = nullptr;
    float* sys_theta2 = nullptr;
    int32_t* sys_heavy = nullptr;
    float* sys_bbox = nullptr;      // [nsys][4]
    uint32_t* sys_maxleaf = nullptr;
    uint32_t* sys_sort_offs = nullptr;  // digit starts of the system sort passes
    int sys_passes = 1;
    uint4* blk = nullptr;           // prepare blocks: (system, first, end)
    uint32_t* sys_blk = nullptr;    // [nsys + 1]
    float2* partial = nullptr;
    int nblk = 0;
    float* vtmp = nullptr;          // 3 x total velocity scratch
    cudaGraphExec_t g_force = nullptr, g_step = nullptr;
    bool dirty = true;
    DevArrays cap_arr{};            // arrays the graphs were captured with
    float* cap_v[3] = {nullptr, nullptr, nullptr};
    float cap_dt = 0.f;
    double grid_scale = 1.0;
    int variant = PSG_MORTON_AVX2;
    std::vector<uint32_t> leaf_ladder{1u, 16u, 32u, 64u};  // leaf capacities the autotuner tries
    int order = 0;                     // local expansion: 0 the reference's, 1 order-1
    std::vector<int> order_ladder{0, 1};  // expansion orders the autotuner tries
};

static DevArrays slice(const DevArrays& a, size_t off) {
    DevArrays d = a;
    d.x += off; d.y += off; d.z += off; d.m += off;
    d.fx += off; d.fy += off; d.fz += off; d.id += off; d.codes += off;
    return d;
}

static int ensure_tick_scratch(State* s) {
    if (s->tk_bbox) return PSG_OK;
    s->tk_grid = s->sms * 4;
    PSG_ALLOC(s->tk_partial, s->tk_grid * sizeof(float2));
    PSG_ALLOC(s->tk_bbox, 4 * sizeof(float));
    for (int c = 0; c < 3; ++c) PSG_ALLOC(s->tk_v[c], s->max_particles * 4);
    for (int c = 0; c < 3; ++c) PSG_ALLOC(s->tk_vmir[c], s->max_particles * 4);
    return PSG_OK;
}

// the local expansion of a state's traversal: 0 the reference's order 0,
// 1 the order-1 expansion (closure mode 1: its field gradients per node)
static int set_order(State* s, int order) {
    if (order >= 1) {
        const int r = closure_alloc(s);
        if (r != PSG_OK) return r;
    }
    s->cl.mode = order >= 1 ? 1 : 0;
    s->order = order >= 1 ? 1 : 0;
    reset_near_levels(s);
    return PSG_OK;
}

// theta, theta^2 (rounded as the MAC rounds it), shallow-leaf depth and leaf
// capacity of every system to the device tables
static int upload_systems(Ensemble* e) {
    std::vector<float> th2(e->nsys);
    std::vector<int32_t> hv(e->nsys);
    int hmax = 0;
    for (size_t k = 0; k < e->nsys; ++k) {
        const float t = e->theta[k];
        th2[k] = t * t;
        hv[k] = heavy_depth_of(t, e->count[k]);
        hmax = std::max(hmax, (int)hv[k]);
    }
    PSG_CHECK(cudaMemcpy(e->sys_theta2, th2.data(), e->nsys * 4, cudaMemcpyHostToDevice));
    PSG_CHECK(cudaMemcpy(e->sys_heavy, hv.data(), e->nsys * 4, cudaMemcpyHostToDevice));
    PSG_CHECK(cudaMemcpy(e->sys_cap, e->cap.data(), e->nsys * 4, cudaMemcpyHostToDevice));
    if (hmax != e->fs->forest_heavy) e->dirty = true;  // a launch parameter changes
    e->fs->forest_heavy = hmax;
    // the stores' near-list depth and P2P mode start over with the settings
    // (both are launch parameters of the captured graphs)
    if (e->fs->ns_levels != kMaxDepth || e->fs->stream_p2p) e->dirty = true;
    e->fs->ns_levels = kMaxDepth;
    e->fs->stream_p2p = 0;
    return PSG_OK;
}

static void drop_graphs(Ensemble* e) {
    if (e->g_force) cudaGraphExecDestroy(e->g_force);
    if (e->g_step) cudaGraphExecDestroy(e->g_step);
    e->g_force = e->g_step = nullptr;
    e->dirty = true;
}

// one tick's forces of all systems, enqueued on the forest stream without
// any host synchronisation (capturable)
static int enqueue_forest_forces(Ensemble* e, const DevArrays& d) {
    State* s = e->fs;
    cudaStream_t st = s->stream;
    const size_t n = e->total;
    const int g = grid_for(s, n, 1024);
    launch_forest_reset_ids(d.id, n, e->part_sys, e->sys_off, g, st);
    launch_prepare_forest(d.x, d.y, d.z, e->blk, e->nblk, e->sys_blk, e->sys_off, e->partial,
                          d.codes, e->sys_bbox, e->variant, st);
    PSG_CHECK(cudaMemsetAsync(s->d_status, 0, sizeof(Status), st));
    PSG_CHECK(cudaMemsetAsync(e->sys_maxleaf, 0, e->nsys * 4, st));
    launch_sort_forest(s->sort, d.codes, n, g, s->d_status, st, e->part_sys, e->sys_passes,
                       e->sys_sort_offs);
    launch_gather(s->sort.perm, d.x, d.y, d.z, d.m, d.id, n, s->xyzm, s->ids, g, st);
    launch_writeback(s->xyzm, s->ids, n, d.x, d.y, d.z, d.m, d.id, g, st);
    const int gt = (int)((s->tv.lvl_base[kLevels] + 255) / 256);
    launch_tree(d.codes, n, s->tree_tiles, s->tv, s->d_status, 0.f, 0.f, 0.f, 0.f, gt, st,
                nullptr, 1);
    launch_upward(s->tv, s->d_status, s->xyzm, gt, st);
    s->trav_n = n;
    int r = enqueue_traversal(s, s->xyzm, d.fx, d.fy, d.fz);
    if (r != PSG_OK) return r;
    launch_forest_single_forces(e->sys_off, (uint32_t)e->nsys, d.fx, d.fy, d.fz, st);
    PSG_CHECK(cudaMemcpyAsync(s->h_status, s->d_status, sizeof(Status), cudaMemcpyDeviceToHost,
                              st));
    return PSG_OK;
}

// every system's velocity permutation through its ids + semi-implicit Euler
static int enqueue_forest_step(Ensemble* e, const DevArrays& d, float* const v[3], float dt) {
    State* s = e->fs;
    cudaStream_t st = s->stream;
    const size_t n = e->total;
    TickState ts;
    ts.id = d.id;
    ts.vx_in = v[0]; ts.vy_in = v[1]; ts.vz_in = v[2];
    ts.vx_out = e->vtmp; ts.vy_out = e->vtmp + n; ts.vz_out = e->vtmp + 2 * n;
    ts.x = d.x; ts.y = d.y; ts.z = d.z; ts.m = d.m;
    ts.fx = d.fx; ts.fy = d.fy; ts.fz = d.fz;
    launch_forest_euler(ts, n, dt, e->part_sys, e->sys_off, grid_for(s, n, 1024), st);
    for (int c = 0; c < 3; ++c)
        PSG_CHECK(cudaMemcpyAsync(v[c], e->vtmp + c * n, n * 4, cudaMemcpyDeviceToDevice, st));
    return PSG_OK;
}

static int capture(Ensemble* e, bool forces, const DevArrays& a, float* const v[3], float dt,
                   cudaGraphExec_t* out) {
    cudaStream_t st = e->fs->stream;
    PSG_CHECK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    int r = forces ? enqueue_forest_forces(e, a) : enqueue_forest_step(e, a, v, dt);
    cudaGraph_t graph = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(st, &graph);
    if (r == PSG_OK && ce != cudaSuccess) {
        note("cudaStreamEndCapture", ce);
        r = PSG_EDEVICE;
    }
    if (r == PSG_OK) {
        const cudaError_t ie = cudaGraphInstantiate(out, graph, 0ull);
        if (ie != cudaSuccess) {
            note("cudaGraphInstantiate", ie);
            r = PSG_EDEVICE;
        }
    }
    if (graph) cudaGraphDestroy(graph);
    return r;
}

static int ensure_graphs(Ensemble* e, const DevArrays& a, float* const v[3], float dt) {
    const bool same = !e->dirty && std::memcmp(&e->cap_arr, &a, sizeof(DevArrays)) == 0 &&
                      e->cap_v[0] == v[0] && e->cap_v[1] == v[1] && e->cap_v[2] == v[2] &&
                      e->cap_dt == dt;
    if (same) return PSG_OK;
    drop_graphs(e);
    e->fs->grid_scale = e->grid_scale;
    int r = capture(e, true, a, v, dt, &e->g_force);
    if (r == PSG_OK) r = capture(e, false, a, v, dt, &e->g_step);
    if (r != PSG_OK) {
        drop_graphs(e);
        return r;
    }
    e->cap_arr = a;
    for (int c = 0; c < 3; ++c) e->cap_v[c] = v[c];
    e->cap_dt = dt;
    e->dirty = false;
    return PSG_OK;
}

// after a forces replay: fatal status -> error; capacity bits -> regrow and
// rerun the traversal, and capture again before the next tick
static int check_forest(Ensemble* e, const DevArrays& a) {
    State* s = e->fs;
    const uint32_t err = s->h_status->err;
    if (err & (PSG_ERR_SORT_SPIN | PSG_ERR_STACK | PSG_ERR_NODES | PSG_ERR_CHAIN_ORDER)) {
        std::snprintf(g_err, sizeof(g_err), "ensemble: device status 0x%x", err);
        return (err & PSG_ERR_NODES) ? PSG_EINVAL : PSG_EDEVICE;
    }
    if (err & (PSG_ERR_NS_OVERFLOW | PSG_ERR_P2P_OVERFLOW | PSG_ERR_DENSE_OVERFLOW |
               PSG_ERR_HEAVY_OVERFLOW)) {
        int r = regrow(s, err);
        if (r != PSG_OK) return r;
        PSG_CHECK(cudaMemsetAsync(&s->d_status->err, 0, 4, s->stream));
        uint32_t err2 = 0;
        r = run_traversal(s, s->xyzm, a.fx, a.fy, a.fz, &err2);
        if (r != PSG_OK) return r;
        if (err2 & (PSG_ERR_SORT_SPIN | PSG_ERR_STACK | PSG_ERR_NODES | PSG_ERR_CHAIN_ORDER |
                    PSG_ERR_HEAVY_OVERFLOW)) {
            std::snprintf(g_err, sizeof(g_err), "ensemble: device status 0x%x", err2);
            return PSG_EDEVICE;
        }
        e->dirty = true;
    }
    return PSG_OK;
}

static int ens_map(Ensemble* e, const psg_arrays_t* a, DevArrays& d) {
    if (a->n != e->total) {
        std::snprintf(g_err, sizeof(g_err), "ensemble: %zu particles given, %zu expected", a->n,
                      e->total);
        return PSG_EINVAL;
    }
    d.x = a->x; d.y = a->y; d.z = a->z; d.m = a->mass;
    d.fx = a->fx; d.fy = a->fy; d.fz = a->fz; d.id = a->id; d.codes = a->codes;
    void* ps[9] = {d.x, d.y, d.z, d.m, d.fx, d.fy, d.fz, d.id, d.codes};
    for (void* p : ps) {
        if (!on_device(p)) {
            std::snprintf(g_err, sizeof(g_err), "ensemble arrays must be device memory");
            return PSG_EINVAL;
        }
    }
    d.any_host = false;
    return PSG_OK;
}

static void free_ensemble(Ensemble* e) {
    if (e->fs && e->fs->stream) cudaStreamSynchronize(e->fs->stream);
    drop_graphs(e);
    if (e->fs) {
        if (e->fs->magic == kMagic) free_state(e->fs);
        delete e->fs;
        e->fs = nullptr;
    }
    void* ps[] = {e->part_sys, e->sys_off, e->sys_cap, e->sys_theta2, e->sys_heavy,
                  e->sys_bbox, e->sys_maxleaf, e->sys_sort_offs, e->blk, e->sys_blk,
                  e->partial, e->vtmp};
    for (void* p : ps)
        if (p) cudaFree(p);
    e->magic = 0;
}

static int ens_create(Ensemble* e, const size_t* counts, size_t nsys, const float* theta) {
    PSG_CHECK(cudaGetDevice(&e->device));
    e->nsys = nsys;
    e->count.assign(counts, counts + nsys);
    e->offset.resize(nsys);
    size_t off = 0;
    for (size_t k = 0; k < nsys; ++k) {
        e->offset[k] = off;
        off += counts[k];
    }
    e->total = off;
    if (off >= 0xFFFFFFF0ull || nsys > 65536) {
        std::snprintf(g_err, sizeof(g_err), "ensemble: at most 65,536 systems and 2^32 particles");
        return PSG_EINVAL;
    }
    e->theta.resize(nsys);
    for (size_t k = 0; k < nsys; ++k) e->theta[k] = theta && theta[k] > 0.f ? theta[k] : 2.0f;
    e->cap.assign(nsys, 1u);
    // level capacities: the sum over systems of min(8^d, N_k); level 0 holds
    // the roots
    uint32_t caps[kLevels];
    for (int d = 0; d <= kMaxDepth; ++d) {
        unsigned long long c = 0;
        for (size_t k = 0; k < nsys; ++k)
            c += d == 0 ? 1ull : std::min<unsigned long long>(1ull << (3 * d), counts[k]);
        if (c >= 0xFFFFFFF0ull) return PSG_EINVAL;
        caps[d] = (uint32_t)c;
    }
    e->sys_passes = nsys > 256 ? 2 : 1;
    e->fs = new (std::nothrow) State;
    if (!e->fs) return PSG_EALLOC;
    int r = init_state(e->fs, e->total, 2.0f, caps, 4 + e->sys_passes);
    if (r != PSG_OK) return r;
    r = ensure_tick_scratch(e->fs);
    if (r != PSG_OK) return r;
    // the shallow-leaf walk serves the shallow groups of every system: more
    // blocks, each frontier sized for the largest system
    {
        size_t maxn = 1;
        for (size_t k = 0; k < nsys; ++k) maxn = std::max(maxn, counts[k]);
        e->fs->heavy_slots = e->fs->sms * 2;
        r = alloc_heavy(e->fs, (uint32_t)(maxn / 4 + 4096));
        if (r != PSG_OK) return r;
    }
    // per-system tables
    std::vector<uint32_t> psys(e->total), soff(nsys + 1), sblk(nsys + 1);
    std::vector<uint4> blk;
    for (size_t k = 0; k < nsys; ++k) {
        soff[k] = (uint32_t)e->offset[k];
        sblk[k] = (uint32_t)blk.size();
        for (size_t i = 0; i < counts[k]; ++i) psys[e->offset[k] + i] = (uint32_t)k;
        for (size_t b = 0; b < counts[k]; b += kForestBlock)
            blk.push_back(make_uint4((uint32_t)k, (uint32_t)(e->offset[k] + b),
                                     (uint32_t)(e->offset[k] + std::min<size_t>(b + kForestBlock,
                                                                               counts[k])),
                                     0u));
    }
    soff[nsys] = (uint32_t)e->total;
    sblk[nsys] = (uint32_t)blk.size();
    e->nblk = (int)blk.size();
    // digit starts of the system passes: the systems are contiguous, so a
    // digit's start is where its first system starts (low byte pass: systems
    // grouped by their low byte)
    std::vector<uint32_t> so(256 * e->sys_passes, 0u);
    for (int q = 0; q < e->sys_passes; ++q) {
        std::vector<unsigned long long> hist(256, 0ull);
        for (size_t k = 0; k < nsys; ++k) hist[(k >> (8 * q)) & 0xFFu] += counts[k];
        unsigned long long run = 0;
        for (int dgt = 0; dgt < 256; ++dgt) {
            so[256 * q + dgt] = (uint32_t)run;
            run += hist[dgt];
        }
    }
    PSG_ALLOC(e->part_sys, e->total * 4);
    PSG_ALLOC(e->sys_off, (nsys + 1) * 4);
    PSG_ALLOC(e->sys_cap, nsys * 4);
    PSG_ALLOC(e->sys_theta2, nsys * 4);
    PSG_ALLOC(e->sys_heavy, nsys * 4);
    PSG_ALLOC(e->sys_bbox, nsys * 16);
    PSG_ALLOC(e->sys_maxleaf, nsys * 4);
    PSG_ALLOC(e->sys_sort_offs, so.size() * 4);
    PSG_ALLOC(e->blk, blk.size() * sizeof(uint4));
    PSG_ALLOC(e->sys_blk, (nsys + 1) * 4);
    PSG_ALLOC(e->partial, blk.size() * sizeof(float2));
    PSG_ALLOC(e->vtmp, 3 * e->total * sizeof(float));
    PSG_CHECK(cudaMemcpy(e->part_sys, psys.data(), e->total * 4, cudaMemcpyHostToDevice));
    PSG_CHECK(cudaMemcpy(e->sys_off, soff.data(), (nsys + 1) * 4, cudaMemcpyHostToDevice));
    PSG_CHECK(cudaMemcpy(e->sys_sort_offs, so.data(), so.size() * 4, cudaMemcpyHostToDevice));
    PSG_CHECK(cudaMemcpy(e->blk, blk.data(), blk.size() * sizeof(uint4), cudaMemcpyHostToDevice));
    PSG_CHECK(cudaMemcpy(e->sys_blk, sblk.data(), (nsys + 1) * 4, cudaMemcpyHostToDevice));
    TreeView& tv = e->fs->tv;
    tv.part_sys = e->part_sys;
    tv.sys_off = e->sys_off;
    tv.sys_cap = e->sys_cap;
    tv.sys_bbox = e->sys_bbox;
    tv.sys_theta2 = e->sys_theta2;
    tv.sys_heavy = e->sys_heavy;
    tv.sys_maxleaf = e->sys_maxleaf;
    tv.nsys = (uint32_t)nsys;
    r = upload_systems(e);
    if (r != PSG_OK) return r;
    e->magic = kEnsMagic;
    return PSG_OK;
}

static int ens_run(Ensemble* e, const psg_arrays_t* a, float* const v[3], float dt,
                   uint32_t ticks) {
    DevArrays d;
    int r = ens_map(e, a, d);
    if (r != PSG_OK) return r;
    for (int c = 0; c < 3; ++c) {
        if (!on_device(v[c])) {
            std::snprintf(g_err, sizeof(g_err), "ensemble velocities must be device memory");
            return PSG_EINVAL;
        }
    }
    PSG_CHECK(cudaSetDevice(e->device));
    cudaStream_t st = e->fs->stream;
    for (uint32_t t = 0; t < ticks; ++t) {
        r = ensure_graphs(e, d, v, dt);
        if (r != PSG_OK) return r;
        PSG_CHECK(cudaGraphLaunch(e->g_force, st));
        PSG_CHECK(cudaStreamSynchronize(st));
        r = check_forest(e, d);
        if (r != PSG_OK) return r;
        PSG_CHECK(cudaGraphLaunch(e->g_step, st));
    }
    PSG_CHECK(cudaStreamSynchronize(st));
    return PSG_OK;
}

// Autotuner.  Per size class (the systems with the same floor(log2 N)) and
// per leaf capacity of its ladder: the smallest theta of {1, 1.5, 2, 3, 4, 6,
// 8} whose median relative force error against an FP64 direct sum on up to
// 1024 particles of the class's first system is at most `target` (a tick of
// that system alone).  Then, class by class from the one holding the most
// particles: the leaf capacity (with its theta) whose whole-ensemble forces
// replay is fastest, among those that met the target.  Last, the traversal
// grids' scale among {1, 1/2, 1/4} by the same replay time.  Works on copies;
// the caller's arrays are left as they are.
static int ens_autotune(Ensemble* e, const psg_arrays_t* a, float target, float* theta_out,
                        double* scale_out) {
    DevArrays d;
    int r = ens_map(e, a, d);
    if (r != PSG_OK) return r;
    PSG_CHECK(cudaSetDevice(e->device));
    cudaStream_t st = e->fs->stream;
    const size_t T = e->total;
    float* buf = nullptr;  // scratch copy: x y z m fx fy fz (7 T floats), id, codes
    PSG_ALLOC(buf, (size_t)9 * T * 4 + 16);
    DevArrays c;
    c.x = buf; c.y = buf + T; c.z = buf + 2 * T; c.m = buf + 3 * T;
    c.fx = buf + 4 * T; c.fy = buf + 5 * T; c.fz = buf + 6 * T;
    c.id = (uint32_t*)(buf + 7 * T); c.codes = (uint32_t*)(buf + 8 * T);
    c.any_host = false;
    auto restore = [&]() -> int {
        PSG_CHECK(cudaMemcpyAsync(c.x, d.x, T * 4, cudaMemcpyDeviceToDevice, st));
        PSG_CHECK(cudaMemcpyAsync(c.y, d.y, T * 4, cudaMemcpyDeviceToDevice, st));
        PSG_CHECK(cudaMemcpyAsync(c.z, d.z, T * 4, cudaMemcpyDeviceToDevice, st));
        PSG_CHECK(cudaMemcpyAsync(c.m, d.m, T * 4, cudaMemcpyDeviceToDevice, st));
        PSG_CHECK(cudaStreamSynchronize(st));
        return PSG_OK;
    };
    static const float ladder[] = {1.0f, 1.5f, 2.0f, 3.0f, 4.0f, 6.0f, 8.0f};
    const int nl = (int)(sizeof(ladder) / sizeof(ladder[0]));
    std::vector<int> cls(e->nsys);
    for (size_t k = 0; k < e->nsys; ++k)
        cls[k] = (int)std::floor(std::log2((double)e->count[k] + 1));
    std::vector<int> classes;  // distinct classes, by the particles they hold (most first)
    std::vector<size_t> rep;   // the first system of each class
    {
        std::vector<std::pair<unsigned long long, int>> held;
        for (size_t k = 0; k < e->nsys; ++k) {
            auto it = std::find(classes.begin(), classes.end(), cls[k]);
            if (it == classes.end()) {
                classes.push_back(cls[k]);
                rep.push_back(k);
                held.push_back({0ull, (int)classes.size() - 1});
                it = classes.end() - 1;
            }
            held[it - classes.begin()].first += e->count[k];
        }
        std::sort(held.begin(), held.end(), [](auto& x, auto& y) { return x.first > y.first; });
        std::vector<int> c2;
        std::vector<size_t> r2;
        for (auto& h : held) {
            c2.push_back(classes[h.second]);
            r2.push_back(rep[h.second]);
        }
        classes = c2;
        rep = r2;
    }
    const size_t ncls = classes.size(), nlc = e->leaf_ladder.size();
    const size_t nor = e->order_ladder.size();
    std::vector<std::vector<std::vector<float>>> thx(
        nor, std::vector<std::vector<float>>(nlc, std::vector<float>(ncls, ladder[nl - 1])));
    std::vector<std::vector<std::vector<bool>>> metx(
        nor, std::vector<std::vector<bool>>(nlc, std::vector<bool>(ncls, false)));
    const size_t kSample = 1024;
    uint32_t* d_tg = nullptr;
    double* d_f64 = nullptr;
    PSG_ALLOC(d_tg, kSample * 4);
    PSG_ALLOC(d_f64, kSample * 3 * sizeof(double));
    size_t maxn = 1;
    for (size_t k = 0; k < e->nsys; ++k) maxn = std::max(maxn, e->count[k]);
    const int dsms = e->fs->sms * 8;
    const size_t part_n = direct_f64_part_doubles(maxn, kSample, dsms);
    double* d_part = nullptr;
    PSG_ALLOC(d_part, part_n * sizeof(double));
    std::vector<uint32_t> tg(kSample);
    std::vector<double> f64(kSample * 3);
    // theta per (leaf capacity, class): ticks of the class's first system alone
    for (size_t ci = 0; ci < ncls && r == PSG_OK; ++ci) {
        const size_t k = rep[ci], n = e->count[k];
        State* s = new (std::nothrow) State;
        if (!s) { r = PSG_EALLOC; break; }
        r = init_state(s, n, 2.0f);
        if (r == PSG_OK) r = ensure_tick_scratch(s);
        const DevArrays ck = slice(c, e->offset[k]);
        for (size_t oi = 0; oi < nor && r == PSG_OK; ++oi)
        for (size_t li = 0; li < nlc && r == PSG_OK; ++li) {
            if ((r = set_order(s, e->order_ladder[oi])) != PSG_OK) break;
            auto& th = thx[oi];
            auto& met = metx[oi];
            s->leaf_cap = e->leaf_ladder[li];
            for (int ti = 0; ti < nl && r == PSG_OK; ++ti) {
                s->theta = ladder[ti];
                reset_near_levels(s);
                if ((r = restore()) != PSG_OK) break;
                launch_tick_reset_ids(ck.id, n, grid_for(s, n, 1024), s->stream);
                int gp = (int)((n + 1023) / 1024);
                if (gp > s->tk_grid) gp = s->tk_grid;
                launch_prepare(ck.x, ck.y, ck.z, n, s->tk_partial, gp, ck.codes, s->tk_bbox,
                               e->variant, s->stream);
                if ((r = tick_core(s, ck, n, 0.f, 0.f, 0.f, 0.f, s->tk_bbox)) != PSG_OK) break;
                const size_t ns = n < kSample ? n : kSample;
                for (size_t i = 0; i < ns; ++i) tg[i] = (uint32_t)(i * n / ns);
                PSG_CHECK(cudaMemcpyAsync(d_tg, tg.data(), ns * 4, cudaMemcpyHostToDevice,
                                          s->stream));
                launch_direct_f64(s->xyzm, n, d_tg, ns, d_f64, dsms, s->stream, d_part, part_n);
                PSG_CHECK(cudaMemcpyAsync(f64.data(), d_f64, ns * 3 * sizeof(double),
                                          cudaMemcpyDeviceToHost, s->stream));
                std::vector<float> hf[3] = {std::vector<float>(n), std::vector<float>(n),
                                            std::vector<float>(n)};
                PSG_CHECK(cudaMemcpyAsync(hf[0].data(), ck.fx, n * 4, cudaMemcpyDeviceToHost,
                                          s->stream));
                PSG_CHECK(cudaMemcpyAsync(hf[1].data(), ck.fy, n * 4, cudaMemcpyDeviceToHost,
                                          s->stream));
                PSG_CHECK(cudaMemcpyAsync(hf[2].data(), ck.fz, n * 4, cudaMemcpyDeviceToHost,
                                          s->stream));
                PSG_CHECK(cudaStreamSynchronize(s->stream));
                std::vector<double> rel(ns);
                for (size_t i = 0; i < ns; ++i) {
                    const double gx = f64[3 * i], gy = f64[3 * i + 1], gz = f64[3 * i + 2];
                    const double ex = hf[0][tg[i]] - gx, ey = hf[1][tg[i]] - gy,
                                 ez = hf[2][tg[i]] - gz;
                    const double nr = std::sqrt(gx * gx + gy * gy + gz * gz);
                    rel[i] = nr > 0 ? std::sqrt(ex * ex + ey * ey + ez * ez) / nr : 0.0;
                }
                std::nth_element(rel.begin(), rel.begin() + ns / 2, rel.end());
                if (rel[ns / 2] <= (double)target) {
                    th[li][ci] = ladder[ti];
                    met[li][ci] = true;
                    break;
                }
            }
        }
        if (s->magic == kMagic) free_state(s);
        delete s;
    }
    cudaFree(d_tg);
    cudaFree(d_f64);
    cudaFree(d_part);
    // one forces replay of the copies with the current settings: its time
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    PSG_CHECK(cudaEventCreate(&t0));
    PSG_CHECK(cudaEventCreate(&t1));
    float* vdummy[3] = {c.fx, c.fy, c.fz};
    auto replay = [&](float* ms) -> int {
        int rr = PSG_OK;
        for (int rep2 = 0; rep2 < 2 && rr == PSG_OK; ++rep2) {  // the first grows stores
            if ((rr = restore()) != PSG_OK) break;
            if ((rr = ensure_graphs(e, c, vdummy, 0.f)) != PSG_OK) break;
            PSG_CHECK(cudaEventRecord(t0, st));
            PSG_CHECK(cudaGraphLaunch(e->g_force, st));
            PSG_CHECK(cudaEventRecord(t1, st));
            PSG_CHECK(cudaStreamSynchronize(st));
            if ((rr = check_forest(e, c)) != PSG_OK) break;
            cudaEventElapsedTime(ms, t0, t1);
        }
        return rr;
    };
    // per expansion order: the class-by-class descent below, then the order
    // whose final replay is fastest
    size_t oi = 0;
    auto set_class = [&](size_t ci, size_t li) {
        for (size_t k = 0; k < e->nsys; ++k) {
            if (cls[k] != classes[ci]) continue;
            e->cap[k] = e->leaf_ladder[li];
            e->theta[k] = thx[oi][li][ci];
        }
    };
    std::vector<std::vector<size_t>> picks(nor, std::vector<size_t>(ncls, 0));
    std::vector<double> order_ms(nor, 1e300);
    for (oi = 0; oi < nor && r == PSG_OK; ++oi) {
        const auto& met = metx[oi];
        auto& pick = picks[oi];
        e->order = e->order_ladder[oi];
        if ((r = set_order(e->fs, e->order)) != PSG_OK) break;
        e->dirty = true;
        // start from each class's first leaf capacity that met the target
        for (size_t ci = 0; ci < ncls; ++ci)
            for (size_t li = 0; li < nlc; ++li)
                if (met[li][ci]) {
                    pick[ci] = li;
                    break;
                }
        for (size_t ci = 0; ci < ncls; ++ci) set_class(ci, pick[ci]);
        if ((r = upload_systems(e)) != PSG_OK) break;
        // then class by class the fastest whole replay
        double best = 1e300;
        for (size_t ci = 0; ci < ncls && r == PSG_OK; ++ci) {
            best = 1e300;
            size_t best_li = pick[ci];
            for (size_t li = 0; li < nlc && r == PSG_OK; ++li) {
                if (nlc > 1 && !met[li][ci] && met[pick[ci]][ci]) continue;
                if (nlc == 1 && li != pick[ci]) continue;
                set_class(ci, li);
                if ((r = upload_systems(e)) != PSG_OK) break;
                e->dirty = true;
                float ms = 0.f;
                if ((r = replay(&ms)) != PSG_OK) break;
                if (ms < best) {
                    best = ms;
                    best_li = li;
                }
            }
            pick[ci] = best_li;
            set_class(ci, best_li);
            if (r == PSG_OK) r = upload_systems(e);
        }
        order_ms[oi] = best;
    }
    if (r == PSG_OK) {
        oi = (size_t)(std::min_element(order_ms.begin(), order_ms.end()) - order_ms.begin());
        e->order = e->order_ladder[oi];
        r = set_order(e->fs, e->order);
        for (size_t ci = 0; ci < ncls; ++ci) set_class(ci, picks[oi][ci]);
        if (r == PSG_OK) r = upload_systems(e);
        e->dirty = true;
    }
    // launch shape: the traversal grids' scale
    if (r == PSG_OK) {
        static const double scales[] = {1.0, 0.5, 0.25};
        double best = 1e300, best_scale = 1.0;
        for (double sc : scales) {
            e->grid_scale = sc;
            e->dirty = true;
            float ms = 0.f;
            if ((r = replay(&ms)) != PSG_OK) break;
            if (ms < best) {
                best = ms;
                best_scale = sc;
            }
        }
        e->grid_scale = best_scale;
        drop_graphs(e);
        if (scale_out) *scale_out = best_scale;
        if (theta_out)
            for (size_t k = 0; k < e->nsys; ++k) theta_out[k] = e->theta[k];
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    cudaFree(buf);
    return r;
}

}  // namespace psg

using psg::State;


extern "C" {

size_t psg_state_bytes(void) { return (sizeof(State) + 63) & ~(size_t)63; }

int psg_init(void* mem, size_t max_particles, float theta) {
    State* s = static_cast<State*>(mem);
    int r = psg::init_state(s, max_particles, theta);
    if (r != PSG_OK) psg::free_state(s);
    return r;
}

int psg_destroy(void* mem) {
    State* s = static_cast<State*>(mem);
    if (!s || s->magic != psg::kMagic) return PSG_EINVAL;
    cudaSetDevice(s->device);
    cudaStreamSynchronize(s->stream);
    psg::free_state(s);
    return PSG_OK;
}

int psg_prepare(const psg_arrays_t* a, float* out_min, float* out_max, float* out_range,
                int variant) {
    return psg::prepare(a, out_min, out_max, out_range, variant);
}

int psg_calc(void* mem, const psg_arrays_t* a, float cx, float cy, float cz, float hw) {
    State* s = static_cast<State*>(mem);
    if (!s || s->magic != psg::kMagic) return PSG_EINVAL;
    return psg::calc(s, a, cx, cy, cz, hw);
}

int psg_run_ticks(void* mem, const psg_arrays_t* a, float* vx, float* vy, float* vz, float dt,
                  uint32_t ticks, int variant) {
    State* s = static_cast<State*>(mem);
    if (!s || s->magic != psg::kMagic) return PSG_EINVAL;
    return psg::run_ticks(s, a, vx, vy, vz, dt, ticks, variant);
}

int psg_set_option(void* mem, int key, double value) {
    State* s = static_cast<State*>(mem);
    if (!s || s->magic != psg::kMagic) return PSG_EINVAL;
    switch (key) {
        case PSG_OPT_DEBUG: s->debug = value != 0.0; return PSG_OK;
        case PSG_OPT_THETA:
            s->theta = value > 0.0 ? (float)value : 1.0f;
            psg::reset_near_levels(s);
            return PSG_OK;
        case PSG_OPT_MORTON_VARIANT:
            if (value < 0 || value > 2) return PSG_EINVAL;
            s->morton_variant = (int)value;
            return PSG_OK;
        case PSG_OPT_TIMING: s->timing = value != 0.0; return PSG_OK;
        case PSG_OPT_KAHAN: s->kahan = value != 0.0; return PSG_OK;
        case PSG_OPT_CLOSURE: {
            const int mode = (int)value;
            if (mode < 0 || mode > 2 || (double)mode != value) return PSG_EINVAL;
            if (mode >= 1) {
                PSG_CHECK(cudaSetDevice(s->device));
                const int r = psg::closure_alloc(s);
                if (r != PSG_OK) return r;
            }
            s->cl.mode = mode;
            s->order = mode >= 1 ? 1 : 0;
            psg::reset_near_levels(s);
            return PSG_OK;
        }
        case PSG_OPT_JUDGE: s->cl.judge = value != 0.0; return PSG_OK;
        case PSG_OPT_JUDGE_BLOCKS:
            if (value < 1 || value > 8 || (double)(int)value != value) return PSG_EINVAL;
            s->cl.judge_bps = (int)value;
            return PSG_OK;
        case PSG_OPT_JUDGE_SAMPLES:
            if (value < 64 || value > psg::kJudgeSamples || (double)(int)value != value)
                return PSG_EINVAL;
            s->cl.judge_samples = (int)value;
            return PSG_OK;
        case PSG_OPT_HEAVY_DEPTH:
            if (value > 5) return PSG_EINVAL;
            s->heavy_depth = value < 0 ? -1 : (int)value;
            return PSG_OK;
        case PSG_OPT_LEAF_CAP:
            if (value < 1 || value > PSG_MAX_LEAF_CAP || (double)(int)value != value)
                return PSG_EINVAL;
            s->leaf_cap = (uint32_t)value;
            psg::reset_near_levels(s);
            return PSG_OK;
        case PSG_OPT_NEAR_LEVELS:
            if (value < 2 || value > psg::kMaxDepth || (double)(int)value != value)
                return PSG_EINVAL;
            s->force_ns_levels = (int)value;
            return PSG_OK;
        case PSG_OPT_STREAM: s->force_stream = value != 0.0; return PSG_OK;
        case PSG_OPT_SHRINK_STORES: {
            if (value != 1.0) return PSG_EINVAL;
            PSG_CHECK(cudaSetDevice(s->device));
            PSG_CHECK(cudaStreamSynchronize(s->stream));
            int r = psg::alloc_ns(s, 1024);
            if (r == PSG_OK) r = psg::alloc_p2p(s, 64);
            if (r == PSG_OK) r = psg::alloc_dense(s, 64);
            psg::reset_near_levels(s);
            return r;
        }
        case PSG_OPT_SORT_SPIN:
            if (value < 0 || value > (1 << 22) || (double)(int)value != value) return PSG_EINVAL;
            s->sort_spin_limit = (int)value;
            return PSG_OK;
        default: return PSG_EINVAL;
    }
}

int psg_get_stats(void* mem, uint64_t* out, size_t n_out) {
    State* s = static_cast<State*>(mem);
    if (!s || s->magic != psg::kMagic || !out) return PSG_EINVAL;
    for (size_t i = 0; i < n_out && i < 24; ++i) out[i] = s->stats[i];
    return PSG_OK;
}

int psg_last_timing(void* mem, float* out_ms, size_t n_out) {
    State* s = static_cast<State*>(mem);
    if (!s || s->magic != psg::kMagic || !out_ms) return PSG_EINVAL;
    for (size_t i = 0; i < n_out && i < (size_t)psg::kPhases; ++i) out_ms[i] = s->ms[i];
    return PSG_OK;
}

size_t psg_tree_nodes(void* mem) {
    State* s = static_cast<State*>(mem);
    if (!s || s->magic != psg::kMagic) return 0;
    return s->last_nodes;
}

// canonical table (level-major, Morton order per level) copied to the host
int psg_tree_dump(void* mem, size_t cap, int32_t* depth, uint32_t* start, uint32_t* count,
                  uint32_t* nchild, int32_t* octant, uint32_t* first_child, uint32_t* parent,
                  float* geo, float* mp, float* lt, uint32_t* m2l_cnt, uint32_t* p2p_cnt) {
    State* s = static_cast<State*>(mem);
    if (!s || s->magic != psg::kMagic) return PSG_EINVAL;
    if (cap < s->last_nodes || s->last_nodes == 0) return cap < s->last_nodes ? PSG_EOOM : PSG_OK;
    PSG_CHECK(cudaSetDevice(s->device));
    // global (capacity-strided) ids -> compact level-major ids
    uint32_t cstart[psg::kLevels + 1];
    cstart[0] = 0;
    for (int d = 0; d <= psg::kMaxDepth; ++d) cstart[d + 1] = cstart[d] + s->lvl_count[d];
    auto compact = [&](uint32_t g, int d) -> uint32_t {
        return g - s->tv.lvl_base[d] + cstart[d];
    };
    size_t k = 0;
    for (int d = 0; d <= psg::kMaxDepth; ++d) {
        const uint32_t cnt = s->lvl_count[d];
        const uint32_t b = s->tv.lvl_base[d];
        if (!cnt) continue;
        uint4* inf = new uint4[cnt];
        PSG_CHECK(cudaMemcpy(inf, s->tv.info + b, cnt * 16, cudaMemcpyDeviceToHost));
        PSG_CHECK(cudaMemcpy(geo + 4 * k, s->tv.geo + b, cnt * 16, cudaMemcpyDeviceToHost));
        PSG_CHECK(cudaMemcpy(mp + 4 * k, s->tv.mp + b, cnt * 16, cudaMemcpyDeviceToHost));
        PSG_CHECK(cudaMemcpy(lt + 4 * k, s->tv.lt + b, cnt * 16, cudaMemcpyDeviceToHost));
        PSG_CHECK(cudaMemcpy(parent + k, s->tv.parent + b, cnt * 4, cudaMemcpyDeviceToHost));
        PSG_CHECK(cudaMemcpy(m2l_cnt + k, s->tv.dbg_m2l + b, cnt * 4, cudaMemcpyDeviceToHost));
        PSG_CHECK(cudaMemcpy(p2p_cnt + k, s->tv.dbg_p2p + b, cnt * 4, cudaMemcpyDeviceToHost));
        for (uint32_t i = 0; i < cnt; ++i) {
            depth[k + i] = d;
            start[k + i] = inf[i].x;
            count[k + i] = inf[i].y;
            nchild[k + i] = psg::flags_nchild(inf[i].w);
            octant[k + i] = d ? (int32_t)psg::flags_octant(inf[i].w) : -1;
            first_child[k + i] = nchild[k + i] ? compact(inf[i].z, d + 1) : 0u;
            parent[k + i] = d ? compact(parent[k + i], d - 1) : 0xFFFFFFFFu;
        }
        delete[] inf;
        k += cnt;
    }
    return PSG_OK;
}

// FP64 direct-sum forces (tests/accuracy.c:42-72) for n_t sampled targets;
// x/y/z/mass, targets and out may each be host or device memory.
int psg_direct_f64(void* mem, const psg_arrays_t* a, const uint32_t* targets, size_t n_t,
                   double* out) {
    State* s = static_cast<State*>(mem);
    if (!s || s->magic != psg::kMagic || !a || !targets || !out) return PSG_EINVAL;
    const size_t n = a->n;
    if (n == 0 || n > s->max_particles) return PSG_EINVAL;
    PSG_CHECK(cudaSetDevice(s->device));
    cudaStream_t st = s->stream;
    const float* src[4] = {a->x, a->y, a->z, a->mass};
    float* tmp = nullptr;
    PSG_ALLOC(tmp, n * 4);
    // pack (x, y, z, m) into the context's particle scratch
    for (int c = 0; c < 4; ++c) {
        const float* p = src[c];
        if (!psg::on_device(p)) {
            PSG_CHECK(cudaMemcpyAsync(tmp, p, n * 4, cudaMemcpyHostToDevice, st));
            p = tmp;
        }
        PSG_CHECK(cudaMemcpy2DAsync((char*)s->xyzm + 4 * c, 16, p, 4, 4, n,
                                    cudaMemcpyDeviceToDevice, st));
        PSG_CHECK(cudaStreamSynchronize(st));
    }
    cudaFree(tmp);
    uint32_t* dt = const_cast<uint32_t*>(targets);
    double* dout = out;
    const bool ht = !psg::on_device(targets), ho = !psg::on_device(out);
    if (ht) {
        PSG_ALLOC(dt, n_t * 4);
        PSG_CHECK(cudaMemcpyAsync(dt, targets, n_t * 4, cudaMemcpyHostToDevice, st));
    }
    if (ho) PSG_ALLOC(dout, n_t * 3 * sizeof(double));
    const size_t part_n = psg::direct_f64_part_doubles(n, n_t, s->sms * 8);
    double* part = nullptr;
    PSG_ALLOC(part, part_n * sizeof(double));
    psg::launch_direct_f64(s->xyzm, n, dt, n_t, dout, s->sms * 8, st, part, part_n);
    PSG_CHECK(cudaGetLastError());
    if (ho) PSG_CHECK(cudaMemcpyAsync(out, dout, n_t * 3 * sizeof(double), cudaMemcpyDeviceToHost, st));
    PSG_CHECK(cudaStreamSynchronize(st));
    cudaFree(part);
    if (ht) cudaFree(dt);
    if (ho) cudaFree(dout);
    return PSG_OK;
}

// ---- batched ensemble ------------------------------------------------------------

int psg_ensemble_create(void** out, const size_t* counts, size_t n_systems, const float* theta) {
    if (!out || !counts || n_systems == 0) return PSG_EINVAL;
    for (size_t k = 0; k < n_systems; ++k)
        if (counts[k] == 0 || counts[k] > 60000000u) return PSG_EINVAL;
    psg::Ensemble* e = new (std::nothrow) psg::Ensemble;
    if (!e) return PSG_EALLOC;
    int r = psg::ens_create(e, counts, n_systems, theta);
    if (r != PSG_OK) {
        psg::free_ensemble(e);
        delete e;
        return r;
    }
    *out = e;
    return PSG_OK;
}

int psg_ensemble_destroy(void* h) {
    psg::Ensemble* e = static_cast<psg::Ensemble*>(h);
    if (!e || e->magic != psg::kEnsMagic) return PSG_EINVAL;
    cudaSetDevice(e->device);
    psg::free_ensemble(e);
    delete e;
    return PSG_OK;
}

int psg_ensemble_run(void* h, const psg_arrays_t* a, float* vx, float* vy, float* vz, float dt,
                     uint32_t ticks) {
    psg::Ensemble* e = static_cast<psg::Ensemble*>(h);
    if (!e || e->magic != psg::kEnsMagic || !a || !vx || !vy || !vz) return PSG_EINVAL;
    float* const v[3] = {vx, vy, vz};
    return psg::ens_run(e, a, v, dt, ticks);
}

int psg_ensemble_autotune(void* h, const psg_arrays_t* a, float target, float* theta_out,
                          double* grid_scale_out) {
    psg::Ensemble* e = static_cast<psg::Ensemble*>(h);
    if (!e || e->magic != psg::kEnsMagic || !a || !(target > 0.f)) return PSG_EINVAL;
    return psg::ens_autotune(e, a, target, theta_out, grid_scale_out);
}

int psg_ensemble_systems(void* h, float* theta_out, size_t n) {
    psg::Ensemble* e = static_cast<psg::Ensemble*>(h);
    if (!e || e->magic != psg::kEnsMagic || !theta_out || n != e->nsys) return PSG_EINVAL;
    for (size_t k = 0; k < n; ++k) theta_out[k] = e->theta[k];
    return PSG_OK;
}

int psg_ensemble_leaf_caps(void* h, uint32_t* cap_out, size_t n) {
    psg::Ensemble* e = static_cast<psg::Ensemble*>(h);
    if (!e || e->magic != psg::kEnsMagic || !cap_out || n != e->nsys) return PSG_EINVAL;
    for (size_t k = 0; k < n; ++k) cap_out[k] = e->cap[k];
    return PSG_OK;
}

int psg_ensemble_set_leaf_caps(void* h, const uint32_t* caps, size_t n, int ladder) {
    psg::Ensemble* e = static_cast<psg::Ensemble*>(h);
    if (!e || e->magic != psg::kEnsMagic || !caps || n == 0) return PSG_EINVAL;
    for (size_t k = 0; k < n; ++k)
        if (caps[k] < 1u || caps[k] > (uint32_t)PSG_MAX_LEAF_CAP) return PSG_EINVAL;
    if (ladder) {
        e->leaf_ladder.assign(caps, caps + n);
        return PSG_OK;
    }
    if (n != e->nsys) return PSG_EINVAL;
    PSG_CHECK(cudaSetDevice(e->device));
    for (size_t k = 0; k < n; ++k) e->cap[k] = caps[k];
    e->dirty = true;
    return psg::upload_systems(e);
}

int psg_ensemble_set_order(void* h, int order) {
    psg::Ensemble* e = static_cast<psg::Ensemble*>(h);
    if (!e || e->magic != psg::kEnsMagic || order > 1) return PSG_EINVAL;
    PSG_CHECK(cudaSetDevice(e->device));
    if (order < 0) {
        e->order_ladder = {0, 1};
        return PSG_OK;
    }
    e->order_ladder = {order};
    e->order = order;
    e->dirty = true;
    const int r = psg::set_order(e->fs, order);
    return r == PSG_OK ? psg::upload_systems(e) : r;
}

int psg_ensemble_order(void* h, int* out) {
    psg::Ensemble* e = static_cast<psg::Ensemble*>(h);
    if (!e || e->magic != psg::kEnsMagic || !out) return PSG_EINVAL;
    *out = e->order;
    return PSG_OK;
}

// ---- learned closure ----------------------------------------------------------

int psg_closure_set_weights(void* mem, const float* params, size_t n_params) {
    State* s = static_cast<State*>(mem);
    if (!s || s->magic != psg::kMagic || !params) return PSG_EINVAL;
    if (n_params != (size_t)psg::kMlpParams) {
        std::snprintf(psg::g_err, sizeof(psg::g_err), "closure weights: %zu parameters, want %d",
                      n_params, psg::kMlpParams);
        return PSG_EINVAL;
    }
    PSG_CHECK(cudaSetDevice(s->device));
    int r = psg::closure_alloc(s);
    if (r != PSG_OK) return r;
    PSG_CHECK(cudaMemcpyAsync(s->cl.params, params, n_params * 4, cudaMemcpyHostToDevice,
                              s->stream));
    psg::launch_mlp_pack(s->cl.params, s->cl.packed, s->stream);
    PSG_CHECK(cudaGetLastError());
    PSG_CHECK(cudaStreamSynchronize(s->stream));
    s->cl.have_weights = 1;
    return PSG_OK;
}

int psg_closure_last(void* mem, double* median_base, double* median_mlp, int* used,
                     int* samples) {
    State* s = static_cast<State*>(mem);
    if (!s || s->magic != psg::kMagic) return PSG_EINVAL;
    if (median_base) *median_base = s->cl.last.median_base;
    if (median_mlp) *median_mlp = s->cl.last.median_mlp;
    if (used) *used = s->cl.last.use_mlp;
    if (samples) *samples = s->cl.last.samples;
    return PSG_OK;
}

// features of sorted particles idx[0, k) after a closure tick (host arrays)
int psg_closure_features(void* mem, const uint32_t* idx, size_t k, float* x_out,
                         float* scale_out) {
    State* s = static_cast<State*>(mem);
    if (!s || s->magic != psg::kMagic || !idx || !x_out || !scale_out) return PSG_EINVAL;
    if (!s->cl.valid) {
        std::snprintf(psg::g_err, sizeof(psg::g_err), "closure features need a closure tick");
        return PSG_EINVAL;
    }
    if (k == 0) return PSG_OK;
    PSG_CHECK(cudaSetDevice(s->device));
    cudaStream_t st = s->stream;
    uint32_t* d_idx = nullptr;
    float* d_x = nullptr;
    PSG_ALLOC(d_idx, k * 4);
    PSG_ALLOC(d_x, k * 17 * 4);
    PSG_CHECK(cudaMemcpyAsync(d_idx, idx, k * 4, cudaMemcpyHostToDevice, st));
    psg::TreeView tv = s->tv;
    tv.lg0 = s->cl.lg0;
    tv.lg1 = s->cl.lg1;
    psg::launch_closure_features(tv, s->cl.leaf_of, s->xyzm, s->last_n, d_idx, k, d_x,
                                 d_x + k * 16, st);
    PSG_CHECK(cudaGetLastError());
    PSG_CHECK(cudaMemcpyAsync(x_out, d_x, k * 16 * 4, cudaMemcpyDeviceToHost, st));
    PSG_CHECK(cudaMemcpyAsync(scale_out, d_x + k * 16, k * 4, cudaMemcpyDeviceToHost, st));
    PSG_CHECK(cudaStreamSynchronize(st));
    cudaFree(d_idx);
    cudaFree(d_x);
    return PSG_OK;
}

// Train the closure MLP with Adam on (x, t) pairs (host arrays, n x 16 and
// n x 3), the learning rate decaying from lr along a cosine to 5 % of it.  params (kMlpParams) holds the initial values and receives the
// trained ones; loss_out (epochs) receives each epoch's mean squared error.
int psg_closure_train(void* mem, const float* x, const float* t, size_t n, float* params,
                      uint32_t epochs, uint32_t batch, float lr, uint64_t seed, float* loss_out) {
    State* s = static_cast<State*>(mem);
    if (!s || s->magic != psg::kMagic || !x || !t || !params || n == 0 || batch == 0)
        return PSG_EINVAL;
    PSG_CHECK(cudaSetDevice(s->device));
    cudaStream_t st = s->stream;
    PSG_CHECK(psg::prepare_mlp_grad_kernel());
    const int P = psg::kMlpParams;
    float *d_x = nullptr, *d_t = nullptr, *d_p = nullptr, *d_m = nullptr, *d_v = nullptr,
          *d_g = nullptr, *d_loss = nullptr;
    uint32_t* d_perm = nullptr;
    psg::MlpPacked* d_w = nullptr;
    PSG_ALLOC(d_x, n * 16 * 4);
    PSG_ALLOC(d_t, n * 3 * 4);
    PSG_ALLOC(d_perm, n * 4);
    PSG_ALLOC(d_p, P * 4);
    PSG_ALLOC(d_m, P * 4);
    PSG_ALLOC(d_v, P * 4);
    PSG_ALLOC(d_g, P * 4);
    PSG_ALLOC(d_loss, (epochs ? epochs : 1) * 4);
    PSG_ALLOC(d_w, sizeof(psg::MlpPacked));
    PSG_CHECK(cudaMemcpyAsync(d_x, x, n * 16 * 4, cudaMemcpyHostToDevice, st));
    PSG_CHECK(cudaMemcpyAsync(d_t, t, n * 3 * 4, cudaMemcpyHostToDevice, st));
    PSG_CHECK(cudaMemcpyAsync(d_p, params, P * 4, cudaMemcpyHostToDevice, st));
    PSG_CHECK(cudaMemsetAsync(d_m, 0, P * 4, st));
    PSG_CHECK(cudaMemsetAsync(d_v, 0, P * 4, st));
    PSG_CHECK(cudaMemsetAsync(d_loss, 0, (epochs ? epochs : 1) * 4, st));
    uint32_t* perm = nullptr;
    PSG_CHECK(cudaMallocHost((void**)&perm, n * 4));
    uint64_t rng = seed ^ 0x9E3779B97F4A7C15ull;
    auto next = [&rng]() {  // splitmix64
        uint64_t z = (rng += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    };
    const float beta1 = 0.9f, beta2 = 0.999f, eps = 1e-8f;
    uint64_t step = 0;
    int r = PSG_OK;
    for (uint32_t ep = 0; ep < epochs && r == PSG_OK; ++ep) {
        PSG_CHECK(cudaStreamSynchronize(st));  // perm is reused
        for (size_t i = 0; i < n; ++i) perm[i] = (uint32_t)i;
        for (size_t i = n - 1; i > 0; --i) {
            const size_t j = (size_t)(next() % (i + 1));
            const uint32_t tmp = perm[i];
            perm[i] = perm[j];
            perm[j] = tmp;
        }
        PSG_CHECK(cudaMemcpyAsync(d_perm, perm, n * 4, cudaMemcpyHostToDevice, st));
        // cosine decay of the learning rate over the epochs, to 5 % of lr
        const float lr_ep =
            lr * (0.05f + 0.95f * 0.5f * (1.0f + cosf(3.14159265f * (float)ep / (float)epochs)));
        for (size_t b0 = 0; b0 < n; b0 += batch) {
            const size_t cnt = n - b0 < batch ? n - b0 : batch;
            PSG_CHECK(cudaMemsetAsync(d_g, 0, P * 4, st));
            psg::launch_mlp_pack(d_p, d_w, st);
            psg::launch_mlp_grad(d_x, d_t, d_perm, b0, cnt, d_w, 1.0f / (3.0f * (float)cnt), d_g,
                                 d_loss + ep, st);
            ++step;
            const float bc1 = 1.0f - powf(beta1, (float)step);
            const float bc2 = 1.0f - powf(beta2, (float)step);
            psg::launch_mlp_adam(d_p, d_m, d_v, d_g, P, lr_ep, beta1, beta2, eps, bc1, bc2, st);
        }
        if (cudaGetLastError() != cudaSuccess) r = PSG_EDEVICE;
    }
    if (r == PSG_OK) {
        PSG_CHECK(cudaMemcpyAsync(params, d_p, P * 4, cudaMemcpyDeviceToHost, st));
        if (loss_out && epochs)
            PSG_CHECK(cudaMemcpyAsync(loss_out, d_loss, epochs * 4, cudaMemcpyDeviceToHost, st));
        PSG_CHECK(cudaStreamSynchronize(st));
        if (loss_out)
            for (uint32_t ep = 0; ep < epochs; ++ep) loss_out[ep] /= (float)(3 * n);
    }
    cudaFreeHost(perm);
    void* bufs[] = {d_x, d_t, d_perm, d_p, d_m, d_v, d_g, d_loss, d_w};
    for (void* b : bufs) cudaFree(b);
    if (r != PSG_OK) std::snprintf(psg::g_err, sizeof(psg::g_err), "closure training failed");
    return r;
}

// loss (mean squared error) and its gradient w.r.t. params for one batch of
// n samples (host arrays): the training step's own kernels, no update
int psg_closure_grad(void* mem, const float* x, const float* t, size_t n, const float* params,
                     float* grad_out, float* loss_out) {
    State* s = static_cast<State*>(mem);
    if (!s || s->magic != psg::kMagic || !x || !t || !params || !grad_out || n == 0)
        return PSG_EINVAL;
    PSG_CHECK(cudaSetDevice(s->device));
    cudaStream_t st = s->stream;
    PSG_CHECK(psg::prepare_mlp_grad_kernel());
    const int P = psg::kMlpParams;
    float *d_x = nullptr, *d_t = nullptr, *d_p = nullptr, *d_g = nullptr, *d_loss = nullptr;
    psg::MlpPacked* d_w = nullptr;
    PSG_ALLOC(d_x, n * 16 * 4);
    PSG_ALLOC(d_t, n * 3 * 4);
    PSG_ALLOC(d_p, P * 4);
    PSG_ALLOC(d_g, P * 4);
    PSG_ALLOC(d_loss, 4);
    PSG_ALLOC(d_w, sizeof(psg::MlpPacked));
    PSG_CHECK(cudaMemcpyAsync(d_x, x, n * 16 * 4, cudaMemcpyHostToDevice, st));
    PSG_CHECK(cudaMemcpyAsync(d_t, t, n * 3 * 4, cudaMemcpyHostToDevice, st));
    PSG_CHECK(cudaMemcpyAsync(d_p, params, P * 4, cudaMemcpyHostToDevice, st));
    PSG_CHECK(cudaMemsetAsync(d_g, 0, P * 4, st));
    PSG_CHECK(cudaMemsetAsync(d_loss, 0, 4, st));
    psg::launch_mlp_pack(d_p, d_w, st);
    psg::launch_mlp_grad(d_x, d_t, nullptr, 0, n, d_w, 1.0f / (3.0f * (float)n), d_g, d_loss, st);
    PSG_CHECK(cudaGetLastError());
    PSG_CHECK(cudaMemcpyAsync(grad_out, d_g, P * 4, cudaMemcpyDeviceToHost, st));
    float loss = 0.f;
    PSG_CHECK(cudaMemcpyAsync(&loss, d_loss, 4, cudaMemcpyDeviceToHost, st));
    PSG_CHECK(cudaStreamSynchronize(st));
    if (loss_out) *loss_out = loss / (float)(3 * n);
    void* bufs[] = {d_x, d_t, d_p, d_g, d_loss, d_w};
    for (void* b : bufs) cudaFree(b);
    return PSG_OK;
}

// MLP outputs (n x 8, before scaling) for inputs x (n x 16), host arrays:
// the inference kernel's network on the tensor cores
int psg_closure_forward(void* mem, const float* x, size_t n, const float* params, float* y_out) {
    State* s = static_cast<State*>(mem);
    if (!s || s->magic != psg::kMagic || !x || !params || !y_out || n == 0) return PSG_EINVAL;
    PSG_CHECK(cudaSetDevice(s->device));
    cudaStream_t st = s->stream;
    float *d_x = nullptr, *d_p = nullptr, *d_y = nullptr;
    psg::MlpPacked* d_w = nullptr;
    PSG_ALLOC(d_x, n * 16 * 4);
    PSG_ALLOC(d_p, psg::kMlpParams * 4);
    PSG_ALLOC(d_y, n * 8 * 4);
    PSG_ALLOC(d_w, sizeof(psg::MlpPacked));
    PSG_CHECK(cudaMemcpyAsync(d_x, x, n * 16 * 4, cudaMemcpyHostToDevice, st));
    PSG_CHECK(cudaMemcpyAsync(d_p, params, psg::kMlpParams * 4, cudaMemcpyHostToDevice, st));
    psg::launch_mlp_pack(d_p, d_w, st);
    PSG_CHECK(cudaMemsetAsync(&s->d_status->err, 0, 4, st));
    psg::launch_mlp_forward(d_x, n, d_w, d_y, s->sms, &s->d_status->err, st);
    PSG_CHECK(cudaGetLastError());
    PSG_CHECK(cudaMemcpyAsync(y_out, d_y, n * 8 * 4, cudaMemcpyDeviceToHost, st));
    PSG_CHECK(cudaMemcpyAsync(&s->h_status->err, &s->d_status->err, 4, cudaMemcpyDeviceToHost,
                              st));
    PSG_CHECK(cudaStreamSynchronize(st));
    void* bufs[] = {d_x, d_p, d_y, d_w};
    for (void* b : bufs) cudaFree(b);
    if (s->h_status->err & PSG_ERR_TC_TIMEOUT) {
        std::snprintf(psg::g_err, sizeof(psg::g_err),
                      "closure network: a tensor-core MMA did not complete");
        return PSG_EDEVICE;
    }
    return PSG_OK;
}

// the last closure tick's per-particle correction (sorted order, n x 3)
int psg_closure_correction(void* mem, float* out, size_t n) {
    State* s = static_cast<State*>(mem);
    if (!s || s->magic != psg::kMagic || !out || !s->cl.dF) return PSG_EINVAL;
    if (n != s->last_n || !s->cl.valid) return PSG_EINVAL;
    PSG_CHECK(cudaSetDevice(s->device));
    PSG_CHECK(cudaMemcpy2DAsync(out, 12, s->cl.dF, 16, 12, n, cudaMemcpyDeviceToHost, s->stream));
    PSG_CHECK(cudaStreamSynchronize(s->stream));
    return PSG_OK;
}

const char* psg_last_error(void) { return psg::g_err; }

void psg_set_error(const char* msg) { std::snprintf(psg::g_err, sizeof(psg::g_err), "%s", msg); }

}  // extern "C"
