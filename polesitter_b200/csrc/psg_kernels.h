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
                 cudaStream_t st);
void launch_gather(const uint32_t* perm, const float* x, const float* y, const float* z,
                   const float* m, const uint32_t* id, size_t n, float4* xyzm, uint32_t* ids,
                   int grid, cudaStream_t st);
void launch_writeback(const float4* xyzm, const uint32_t* ids, size_t n, float* x, float* y,
                      float* z, float* m, uint32_t* id, int grid, cudaStream_t st);

// k_tree.cu -- octree build (polesitter.h:906-967) + upward pass (:971-1046)
int tree_tile_size();
void launch_tree(const uint32_t* codes, size_t n, uint32_t* tile_buf, TreeView tv,
                 Status* status, float cx, float cy, float cz, float hw, int grid,
                 cudaStream_t st, const float* bbox = nullptr);
void launch_upward(TreeView tv, const Status* status, const float4* xyzm, int grid,
                   cudaStream_t st);

// k_traverse.cu -- fused MAC / M2L / L2L, and L2P + P2P for the leaves
// (polesitter.h:1050-1146, :1224-1254, :1258-1494)
struct TravArgs;
int traverse_threads();
const void* traverse_kernel_ptr();
const void* traverse_internal_kernel_ptr();
void launch_traverse_internal(const TravArgs& A, int level, int grid, cudaStream_t st);
void launch_traverse_leaves(const TravArgs& A, int grid, cudaStream_t st);


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

// k_direct.cu -- FP64 direct-sum forces for sampled targets (tests/accuracy.c:42-72)
void launch_direct_f64(const float4* xyzm, size_t n, const uint32_t* targets, size_t n_targets,
                       double* out /*[n_targets][3]*/, cudaStream_t st);

}  // namespace psg

#include "psg_common.cuh"

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
};
}  // namespace psg
