// Host-side launchers of the tick's kernels (one .cu file per phase).
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace psg {

struct TreeView;
struct Status;

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
                 cudaStream_t st);
void launch_upward(TreeView tv, const Status* status, const float4* xyzm, int grid,
                   cudaStream_t st);

// k_traverse.cu -- fused M2L / L2L / L2P / P2P (polesitter.h:1050-1494)
struct TravLaunch;
int traverse_threads();
const void* traverse_kernel_ptr();
void launch_traverse_level(const TravLaunch& L, int level, const uint32_t* ns_in,
                           uint32_t* ns_out, int grid, cudaStream_t st);

// k_direct.cu -- FP64 direct-sum forces for sampled targets (tests/accuracy.c:42-72)
void launch_direct_f64(const float4* xyzm, size_t n, const uint32_t* targets, size_t n_targets,
                       double* out /*[n_targets][3]*/, cudaStream_t st);

}  // namespace psg

#include "psg_common.cuh"

namespace psg {
struct TravLaunch {
    TreeView tv;
    const float4* xyzm;
    float* fx;
    float* fy;
    float* fz;
    unsigned long long ns_cap;
    double* facc;
    Status* status;
    float theta;
    int debug;
};
}  // namespace psg
