// ps_prepare_particles on the GPU: the cubic bounding box over x, y, z
// jointly and the 30-bit Morton code of every particle.
//
// Reference: polesitter.h:1911-2170.  Both kernels are HBM-bound streams:
// 12 B/particle read for the box, 12 B read + 4 B written for the codes.
#include "psg_common.cuh"
#include "psg_kernels.h"

namespace psg {

// 10-bit -> 30-bit spread with two zero bits between input bits
// (polesitter.h:778-787).
__device__ __forceinline__ uint32_t expand10(uint32_t v) {
    v &= 0x3FFu;
    v = (v | (v << 16)) & 0x030000FFu;
    v = (v | (v << 8)) & 0x0300F00Fu;
    v = (v | (v << 4)) & 0x030C30C3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

__device__ __forceinline__ uint32_t morton3(uint32_t qx, uint32_t qy, uint32_t qz) {
    return expand10(qx) | (expand10(qy) << 1) | (expand10(qz) << 2);
}

// Lanes of the reference's vector path (polesitter.h:2046-2058):
// q = (v - min) * (1023 / range); q = max(0, min(q, 1023)) with the SSE
// operand order (a NaN becomes 1023); then round-to-nearest-even (AVX2) or
// truncation (NEON, :2111).
__device__ __forceinline__ uint32_t quant_vec(float v, float mn, float scale, bool trunc) {
    float q = __fmul_rn(__fsub_rn(v, mn), scale);
    q = (q < 1023.0f) ? q : 1023.0f;
    q = (0.0f > q) ? 0.0f : q;
    return (uint32_t)(trunc ? __float2int_rz(q) : __float2int_rn(q));
}

// The scalar formula used for the tail that does not fill a vector and for
// scalar builds (polesitter.h:2133-2153).
__device__ __forceinline__ uint32_t quant_scalar(float v, float mn, float range) {
    int q = __float2int_rz(__fmul_rn(__fdiv_rn(__fsub_rn(v, mn), range), 1023.0f));
    q = q < 0 ? 0 : q;
    q = q > 1023 ? 1023 : q;
    return (uint32_t)q;
}

__global__ void __launch_bounds__(256) k_bbox_partial(const float* __restrict__ x,
                                                      const float* __restrict__ y,
                                                      const float* __restrict__ z, size_t n,
                                                      float2* __restrict__ partial) {
    float mn = 3.402823466e38f, mx = -3.402823466e38f;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        float a = __ldg(x + i), b = __ldg(y + i), c = __ldg(z + i);
        mn = fminf(mn, fminf(a, fminf(b, c)));
        mx = fmaxf(mx, fmaxf(a, fmaxf(b, c)));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mn = fminf(mn, __shfl_xor_sync(0xFFFFFFFFu, mn, o));
        mx = fmaxf(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, o));
    }
    __shared__ float2 red[8];
    if (lane_id() == 0) red[threadIdx.x >> 5] = make_float2(mn, mx);
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
            mn = fminf(mn, red[w].x);
            mx = fmaxf(mx, red[w].y);
        }
        partial[blockIdx.x] = make_float2(mn, mx);
    }
}

__global__ void __launch_bounds__(256) k_morton(const float* __restrict__ x,
                                                const float* __restrict__ y,
                                                const float* __restrict__ z, size_t n,
                                                const float2* __restrict__ partial,
                                                int n_partial, uint32_t* __restrict__ codes,
                                                float* __restrict__ bbox_out, int variant) {
    __shared__ float s_box[4];
    if (threadIdx.x < 32) {
        float mn = 3.402823466e38f, mx = -3.402823466e38f;
        for (int i = threadIdx.x; i < n_partial; i += 32) {
            float2 p = partial[i];
            mn = fminf(mn, p.x);
            mx = fmaxf(mx, p.y);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            mn = fminf(mn, __shfl_xor_sync(0xFFFFFFFFu, mn, o));
            mx = fmaxf(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, o));
        }
        if (threadIdx.x == 0) {
            float range = __fsub_rn(mx, mn);  // polesitter.h:2008-2011
            if (range < 0.001f) range = 0.001f;
            s_box[0] = mn;
            s_box[1] = mx;
            s_box[2] = range;
            s_box[3] = __fdiv_rn(1023.0f, range);  // :2017
            if (blockIdx.x == 0 && bbox_out) {
                bbox_out[0] = mn;
                bbox_out[1] = mx;
                bbox_out[2] = range;
                bbox_out[3] = s_box[3];
            }
        }
    }
    __syncthreads();
    const float mn = s_box[0], range = s_box[2], scale = s_box[3];
    const size_t lanes = variant == PSG_MORTON_AVX2 ? 8 : (variant == PSG_MORTON_NEON ? 4 : 0);
    const size_t vec_end = lanes ? (n / lanes) * lanes : 0;
    const bool trunc = (variant == PSG_MORTON_NEON);
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        float a = __ldg(x + i), b = __ldg(y + i), c = __ldg(z + i);
        uint32_t qx, qy, qz;
        if (i < vec_end) {
            qx = quant_vec(a, mn, scale, trunc);
            qy = quant_vec(b, mn, scale, trunc);
            qz = quant_vec(c, mn, scale, trunc);
        } else {
            qx = quant_scalar(a, mn, range);
            qy = quant_scalar(b, mn, range);
            qz = quant_scalar(c, mn, range);
        }
        codes[i] = morton3(qx, qy, qz);
    }
}

// ---- many systems in one array (the batched ensemble) ----
// Block b covers the particles [blk[b].y, blk[b].z) of system blk[b].x; the
// blocks of system k are [sys_blk[k], sys_blk[k + 1]).  Each system gets its
// own box and codes exactly as its own ps_prepare_particles computes them
// (min/max are exact in any order; the vector/tail split is per system).
__global__ void __launch_bounds__(256) k_forest_bbox(const float* __restrict__ x,
                                                     const float* __restrict__ y,
                                                     const float* __restrict__ z,
                                                     const uint4* __restrict__ blk,
                                                     float2* __restrict__ partial) {
    const uint4 b = blk[blockIdx.x];
    float mn = 3.402823466e38f, mx = -3.402823466e38f;
    for (uint32_t i = b.y + threadIdx.x; i < b.z; i += blockDim.x) {
        float a = __ldg(x + i), c = __ldg(y + i), d = __ldg(z + i);
        mn = fminf(mn, fminf(a, fminf(c, d)));
        mx = fmaxf(mx, fmaxf(a, fmaxf(c, d)));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mn = fminf(mn, __shfl_xor_sync(0xFFFFFFFFu, mn, o));
        mx = fmaxf(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, o));
    }
    __shared__ float2 red[8];
    if (lane_id() == 0) red[threadIdx.x >> 5] = make_float2(mn, mx);
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
            mn = fminf(mn, red[w].x);
            mx = fmaxf(mx, red[w].y);
        }
        partial[blockIdx.x] = make_float2(mn, mx);
    }
}

__global__ void __launch_bounds__(256) k_forest_morton(const float* __restrict__ x,
                                                       const float* __restrict__ y,
                                                       const float* __restrict__ z,
                                                       const uint4* __restrict__ blk,
                                                       const uint32_t* __restrict__ sys_blk,
                                                       const uint32_t* __restrict__ sys_off,
                                                       const float2* __restrict__ partial,
                                                       uint32_t* __restrict__ codes,
                                                       float* __restrict__ sys_bbox,
                                                       int variant) {
    const uint4 b = blk[blockIdx.x];
    const uint32_t k = b.x;
    __shared__ float s_box[4];
    if (threadIdx.x < 32) {
        float mn = 3.402823466e38f, mx = -3.402823466e38f;
        for (uint32_t i = sys_blk[k] + threadIdx.x; i < sys_blk[k + 1]; i += 32) {
            float2 p = partial[i];
            mn = fminf(mn, p.x);
            mx = fmaxf(mx, p.y);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            mn = fminf(mn, __shfl_xor_sync(0xFFFFFFFFu, mn, o));
            mx = fmaxf(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, o));
        }
        if (threadIdx.x == 0) {
            float range = __fsub_rn(mx, mn);  // polesitter.h:2008-2011
            if (range < 0.001f) range = 0.001f;
            s_box[0] = mn;
            s_box[1] = mx;
            s_box[2] = range;
            s_box[3] = __fdiv_rn(1023.0f, range);  // :2017
            if (blockIdx.x == sys_blk[k]) {
                sys_bbox[4 * k + 0] = mn;
                sys_bbox[4 * k + 1] = mx;
                sys_bbox[4 * k + 2] = range;
                sys_bbox[4 * k + 3] = s_box[3];
            }
        }
    }
    __syncthreads();
    const float mn = s_box[0], range = s_box[2], scale = s_box[3];
    const uint32_t lo = sys_off[k], n = sys_off[k + 1] - lo;
    const uint32_t lanes = variant == PSG_MORTON_AVX2 ? 8 : (variant == PSG_MORTON_NEON ? 4 : 0);
    const uint32_t vec_end = lanes ? (n / lanes) * lanes : 0;
    const bool trunc = (variant == PSG_MORTON_NEON);
    for (uint32_t i = b.y + threadIdx.x; i < b.z; i += blockDim.x) {
        float a = __ldg(x + i), c = __ldg(y + i), d = __ldg(z + i);
        uint32_t qx, qy, qz;
        if (i - lo < vec_end) {
            qx = quant_vec(a, mn, scale, trunc);
            qy = quant_vec(c, mn, scale, trunc);
            qz = quant_vec(d, mn, scale, trunc);
        } else {
            qx = quant_scalar(a, mn, range);
            qy = quant_scalar(c, mn, range);
            qz = quant_scalar(d, mn, range);
        }
        codes[i] = morton3(qx, qy, qz);
    }
}

void launch_prepare_forest(const float* x, const float* y, const float* z, const uint4* blk,
                           int nblk, const uint32_t* sys_blk, const uint32_t* sys_off,
                           float2* partial, uint32_t* codes, float* sys_bbox, int variant,
                           cudaStream_t st) {
    k_forest_bbox<<<nblk, 256, 0, st>>>(x, y, z, blk, partial);
    k_forest_morton<<<nblk, 256, 0, st>>>(x, y, z, blk, sys_blk, sys_off, partial, codes,
                                          sys_bbox, variant);
}

void launch_prepare(const float* x, const float* y, const float* z, size_t n,
                    float2* partial, int grid, uint32_t* codes, float* bbox_out,
                    int variant, cudaStream_t st) {
    k_bbox_partial<<<grid, 256, 0, st>>>(x, y, z, n, partial);
    k_morton<<<grid, 256, 0, st>>>(x, y, z, n, partial, grid, codes, bbox_out, variant);
}

}  // namespace psg
