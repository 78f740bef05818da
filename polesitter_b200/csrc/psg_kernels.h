// Host-side launchers of the tick's kernels (one .cu file per phase).
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace psg {

struct TreeView;
struct Status;
struct P2PStore;

// k_prepare.cu -- bbox + Morton codes (polesitter.h:1911-2170)
void launch_prepare(const float* x, const float* y, const float* z, size_t n, float2* partial,
                    int grid, uint32_t* codes, float* bbox_out, int variant, cudaStream_t st);
// many systems in one array: block b covers particles [blk[b].y, blk[b].z) of
// system blk[b].x, the blocks of system k are [sys_blk[k], sys_blk[k + 1]);
// sys_bbox receives (min, max, range, 1023 / range) per system
void launch_prepare_forest(const float* x, const float* y, const float* z, const uint4* blk,
                           int nblk, const uint32_t* sys_blk, const uint32_t* sys_off,
                           float2* partial, uint32_t* codes, float* sys_bbox, int variant,
                           cudaStream_t st);

// k_sort.cu -- stable LSD radix sort + gather (polesitter.h:1588-1693)
struct SortBuffers {
    uint32_t* key_a;
    uint32_t* key_b;
    uint32_t* val_a;
    uint32_t* val_b;
    uint32_t* hist;      // [4][256]
    uint32_t* offs;      // [4][256]
    uint32_t* lookback;  // [4][tiles][256]
    uint32_t* perm;      // output: val_a after the last pass
};
int sort_tile_size();
void launch_sort(SortBuffers& b, uint32_t* codes, size_t n, int grid, Status* status,
                 cudaStream_t st, int spin_limit = 0);
// many systems in one array: each sorted within its range (sys_passes stable
// passes on the system index after the code passes; lookback sized for 4 +
// sys_passes passes)
void launch_sort_forest(SortBuffers& b, uint32_t* codes, size_t n, int grid, Status* status,
                        cudaStream_t st, const uint32_t* part_sys, int sys_passes,
                        const uint32_t* sys_offs);
void launch_gather(const uint32_t* perm, const float* x, const float* y, const float* z,
                   const float* m, const uint32_t* id, size_t n, float4* xyzm, uint32_t* ids,
                   int grid, cudaStream_t st);
void launch_writeback(const float4* xyzm, const uint32_t* ids, size_t n, float* x, float* y,
                      float* z, float* m, uint32_t* id, int grid, cudaStream_t st);

// k_tree.cu -- octree build (polesitter.h:906-967) + upward pass (:971-1046)
int tree_tile_size();
void launch_tree(const uint32_t* codes, size_t n, uint32_t* tile_buf, TreeView tv,
                 Status* status, float cx, float cy, float cz, float hw, int grid,
                 cudaStream_t st, const float* bbox = nullptr, uint32_t leaf_cap = 1);
void launch_upward(TreeView tv, const Status* status, const float4* xyzm, int grid,
                   cudaStream_t st);

// k_traverse.cu -- fused MAC / M2L / L2L, and L2P + P2P for the leaves
// (polesitter.h:1050-1146, :1224-1254, :1258-1494)
struct TravArgs;
int traverse_threads();
const void* traverse_kernel_ptr(int order, int dense, int xl);
const void* traverse_internal_kernel_ptr(int order);
void launch_traverse_internal(const TravArgs& A, int level, int grid, cudaStream_t st);
void launch_traverse_leaves(const TravArgs& A, const int grid[2], cudaStream_t st);
void launch_dense_p2p(const TravArgs& A, int grid, cudaStream_t st);
void launch_heavy_leaf(const TravArgs& A, int grid, cudaStream_t st);
void launch_leaf_start(Status* status, int heavy_depth, int order, cudaStream_t st);


// k_tick.cu -- the caller's tick loop on the device (README.md:65-111)
struct TickState {
    const uint32_t* id;   // sorted -> pre-sort index, from this tick's sort
    const float* vx_in;   // velocities in the previous tick's order
    const float* vy_in;
    const float* vz_in;
    float* vx_out;        // velocities in this tick's (sorted) order
    float* vy_out;
    float* vz_out;
    float* x;             // sorted positions, advanced in place
    float* y;
    float* z;
    const float* m;
    const float* fx;
    const float* fy;
    const float* fz;
};
void launch_tick_reset_ids(uint32_t* id, size_t n, int grid, cudaStream_t st);
void launch_tick_euler(const TickState& t, size_t n, float dt, int grid, cudaStream_t st);
// many systems in one array (system k at [sys_off[k], sys_off[k + 1]))
void launch_forest_reset_ids(uint32_t* id, size_t n, const uint32_t* part_sys,
                             const uint32_t* sys_off, int grid, cudaStream_t st);
void launch_forest_euler(const TickState& t, size_t n, float dt, const uint32_t* part_sys,
                         const uint32_t* sys_off, int grid, cudaStream_t st);
void launch_forest_single_forces(const uint32_t* sys_off, uint32_t nsys, float* fx, float* fy,
                                 float* fz, cudaStream_t st);

// k_closure.cu -- the learned far-field closure (no counterpart in the reference)
struct MlpPacked;
struct JudgeOut;
// the network's inference on the tensor cores (tcgen05); err receives
// PSG_ERR_TC_TIMEOUT if an MMA does not complete
void launch_closure_mlp(const TreeView& tv, const uint32_t* leaf_of, const float4* xyzm, size_t n,
                        const MlpPacked* w, float4* dF, int sms, uint32_t* err, cudaStream_t st);
void launch_closure_features(const TreeView& tv, const uint32_t* leaf_of, const float4* xyzm,
                             size_t n, const uint32_t* idx, size_t k, float* x_out,
                             float* scale_out, cudaStream_t st);
// the judge's FP64 direct sum on a sample (runs beside the tree build and
// traversal on its own stream) and its decision (after the traversal)
void launch_judge_direct(const float4* xyzm, size_t n, uint32_t* tg, int s, double* f64,
                         uint32_t tick, int blocks, cudaStream_t st, double* part,
                         size_t part_doubles);
void launch_judge_decide(const uint32_t* tg, int s, const double* f64, const float* fx,
                         const float* fy, const float* fz, const float4* dF, int allow,
                         JudgeOut* out, cudaStream_t st);
void launch_closure_apply(float* fx, float* fy, float* fz, const float4* dF, size_t n,
                          const JudgeOut* j, int sms, cudaStream_t st);
void launch_mlp_pack(const float* params, MlpPacked* out, cudaStream_t st);
void launch_mlp_forward(const float* x, size_t n, const MlpPacked* w, float* y, int sms,
                        uint32_t* err, cudaStream_t st);
cudaError_t prepare_mlp_grad_kernel();
size_t mlp_train_smem_bytes();
void launch_mlp_grad(const float* X, const float* T, const uint32_t* perm, size_t b0,
                     size_t count, const MlpPacked* w, float inv_norm, float* grad,
                     float* loss_sum, cudaStream_t st);
void launch_mlp_adam(float* p, float* m, float* v, const float* g, int n, float lr, float beta1,
                     float beta2, float eps, float bc1, float bc2, cudaStream_t st);

// k_direct.cu -- FP64 direct-sum forces for sampled targets (tests/accuracy.c:42-72)
// part: partial sums of the source splits (summed in split order, so the
// result does not depend on scheduling); as many splits as part_doubles
// holds, at most those that fill about `blocks` blocks
size_t direct_f64_part_doubles(size_t n, size_t n_targets, int blocks);
void launch_direct_f64(const float4* xyzm, size_t n, const uint32_t* targets, size_t n_targets,
                       double* out /*[n_targets][3]*/, int blocks, cudaStream_t st,
                       double* part, size_t part_doubles);

}  // namespace psg

#include "psg_common.cuh"

namespace psg {
// k_dense_p2p: blocks per SM, warps per block, and the partial entries
// (source leaves that serve only some leaves of a record) a warp keeps for
// its record's second pass
constexpr int kDenseBlocksPerSm = 8;
constexpr int kDenseWarpsPerBlock = 4;
constexpr uint32_t kDensePartCap = 2048;
}  // namespace psg

namespace psg {
struct TravArgs {
    TreeView tv;
    P2PStore p2p;       // spill chunks of P2P source lists longer than a chunk
    uint32_t* ns;       // near lists of all levels
    unsigned long long ns_cap;
    const float4* xyzm;  // sorted particles
    float* fx;          // output forces, sorted order
    float* fy;
    float* fz;
    Status* status;
    float theta;
    int level;
    int debug;
    int kahan;          // compensated FP32 sums in P2P
    int order;          // closure: 0 = the reference's order-0 local, 1 = order-1
    uint32_t* leaf_of;  // closure: leaf node of each sorted particle (order 1)
    uint4* dense_rec;   // full-leaf P2P work records: leaf | q << 28, chain, first, count
    uint32_t dense_cap;
    uint2* dense_part;  // per warp of k_dense_p2p: kDensePartCap partial entries
    uint32_t dense_part_warps;
    int heavy_depth;    // leaf children of nodes above this depth go to k_heavy_leaf
    uint32_t* heavy_frontier;  // per block: 2 x heavy_fcap candidate slots
    uint32_t heavy_fcap;
    int ns_levels;      // near lists exist for nodes of depth <= ns_levels; deeper
                        // groups walk their ancestor chain (k_traverse.cu)
    int stream;         // 1: P2P summed in the leaf pass as sources are found, no spill
    uint32_t leaf_cap;  // the tree's leaf capacity (one system)
};
}  // namespace psg
