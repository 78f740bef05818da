// FP64 direct-sum forces on the GPU for a sample of target particles: the
// accuracy yardstick every result is reported against.
//
// Reference: direct_reference in tests/accuracy.c:42-72 --
//   F_i = sum_{j != i} m_i m_j d_ij / (|d_ij|^2 + eps2)^{3/2},
// eps2 = the float literal 0.1F widened to double (accuracy.c:12, :57).
// Sources are streamed through shared memory in tiles; each thread owns two
// targets and accumulates in FP64.  Also the closure's per-tick judge.
#include "psg_common.cuh"
#include "psg_kernels.h"

namespace psg {

constexpr int kDirThreads = 128;
constexpr int kDirPer = 2;  // targets per thread

// 1/sqrt(x) in FP64 for x >= 0.1 (softened squared distances): the hardware's
// approximate reciprocal square root (PTX rsqrt.approx.ftz.f64) refined by one
// Newton-Raphson step for x^(-1/2), y <- y + (y/2)(1 - x y^2), which squares
// its relative error: ~1.5e-12 from a 2^-20 seed, ~5e-12 on 1/r^3, far below
// the errors this yardstick measures (1e-7 .. 1e-1) and below the 1e-10 its
// tests hold it to against the CPU's FP64 sum.
__device__ __forceinline__ double rsqrt_newton(double x) {
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    const double t = fma(-x, y * y, 1.0);
    return fma(0.5 * y, t, y);
}

// One block: 256 targets against the sources [src0, src1) of its split
// (blockIdx.y).  The sources of a target are split over many blocks so that a
// sample of a few thousand targets still fills the GPU; each split writes its
// partial sums to its own slice of part (no atomics), and k_direct_sum adds
// the slices in split order, so the result does not depend on scheduling.
__global__ void __launch_bounds__(kDirThreads) k_direct_f64(const float4* __restrict__ xyzm,
                                                            size_t n,
                                                            const uint32_t* __restrict__ targets,
                                                            size_t n_targets, size_t chunk,
                                                            double* __restrict__ part) {
    // the tile is widened to FP64 once per block, not once per pair; each
    // thread owns kDirPer targets, so each tile read serves kDirPer pairs
    __shared__ double4 tile[kDirThreads];
    size_t k[kDirPer];
    bool active[kDirPer];
    double tx[kDirPer], ty[kDirPer], tz[kDirPer], tm[kDirPer];
    double ax[kDirPer], ay[kDirPer], az[kDirPer];
#pragma unroll
    for (int p = 0; p < kDirPer; ++p) {
        k[p] = (size_t)blockIdx.x * (kDirThreads * kDirPer) + (size_t)p * kDirThreads +
               threadIdx.x;
        const uint32_t ti_raw = k[p] < n_targets ? targets[k[p]] : 0u;
        active[p] = k[p] < n_targets && ti_raw < n;
        const float4 t = active[p] ? xyzm[ti_raw] : make_float4(0.f, 0.f, 0.f, 0.f);
        tx[p] = (double)t.x;
        ty[p] = (double)t.y;
        tz[p] = (double)t.z;
        tm[p] = (double)t.w;
        ax[p] = ay[p] = az[p] = 0.0;
    }
    const double eps2 = (double)0.1f;
    const size_t src0 = (size_t)blockIdx.y * chunk;
    const size_t src1 = src0 + chunk < n ? src0 + chunk : n;
    for (size_t j0 = src0; j0 < src1; j0 += kDirThreads) {
        const size_t j = j0 + threadIdx.x;
        const float4 sj = j < src1 ? xyzm[j] : make_float4(0.f, 0.f, 0.f, 0.f);
        tile[threadIdx.x] = make_double4((double)sj.x, (double)sj.y, (double)sj.z, (double)sj.w);
        __syncthreads();
        const int cnt = (int)((src1 - j0) < (size_t)kDirThreads ? (src1 - j0) : kDirThreads);
        for (int q = 0; q < cnt; ++q) {
            const double4 s = tile[q];
#pragma unroll
            for (int p = 0; p < kDirPer; ++p) {
                const double dx = s.x - tx[p];
                const double dy = s.y - ty[p];
                const double dz = s.z - tz[p];
                const double r2 = fma(dx, dx, fma(dy, dy, fma(dz, dz, eps2)));
                const double ir = rsqrt_newton(r2);
                // the self pair (and any source at the target's position) has
                // d = 0 and adds exactly 0, as j != i excludes it in the sum
                const double w = s.w * ir * ir * ir;
                ax[p] += dx * w;
                ay[p] += dy * w;
                az[p] += dz * w;
            }
        }
        __syncthreads();
    }
    double* out = part + (size_t)blockIdx.y * n_targets * 3;
#pragma unroll
    for (int p = 0; p < kDirPer; ++p) {
        if (k[p] >= n_targets) continue;
        // a target index outside the particles gets NaN (from split 0)
        const double nan = __longlong_as_double(0x7FF8000000000000ll);
        const double bad = blockIdx.y == 0 ? nan : 0.0;
        out[3 * k[p] + 0] = active[p] ? tm[p] * ax[p] : bad;
        out[3 * k[p] + 1] = active[p] ? tm[p] * ay[p] : bad;
        out[3 * k[p] + 2] = active[p] ? tm[p] * az[p] : bad;
    }
}

// out[i] = sum over the splits, in split order
__global__ void k_direct_sum(const double* __restrict__ part, size_t m, int splits,
                             double* __restrict__ out) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) {
        double v = 0.0;
        for (int q = 0; q < splits; ++q) v += part[(size_t)q * m + i];
        out[i] = v;
    }
}

static size_t direct_splits(size_t n, size_t n_targets, int blocks, size_t part_doubles,
                            size_t* chunk_out) {
    const size_t tblocks = (n_targets + kDirThreads * kDirPer - 1) / (kDirThreads * kDirPer);
    // about `blocks` blocks in total, each source chunk at least 1024
    // particles, as many splits as the partial-sum buffer holds
    size_t splits = ((size_t)blocks + tblocks - 1) / tblocks;
    const size_t max_splits = (n + 1023) / 1024;
    if (splits > max_splits) splits = max_splits;
    const size_t fit = part_doubles / (n_targets * 3);
    if (splits > fit) splits = fit;
    if (splits < 1) splits = 1;
    size_t chunk = (n + splits - 1) / splits;
    chunk = (chunk + kDirThreads - 1) / kDirThreads * kDirThreads;
    *chunk_out = chunk;
    return (n + chunk - 1) / chunk;
}

size_t direct_f64_part_doubles(size_t n, size_t n_targets, int blocks) {
    if (n_targets == 0 || n == 0) return 1;
    size_t chunk = 0;
    return direct_splits(n, n_targets, blocks, ~(size_t)0 / 2, &chunk) * n_targets * 3;
}

void launch_direct_f64(const float4* xyzm, size_t n, const uint32_t* targets, size_t n_targets,
                       double* out, int blocks, cudaStream_t st, double* part,
                       size_t part_doubles) {
    if (n_targets == 0) return;
    size_t chunk = 0;
    const size_t splits =
        part ? direct_splits(n, n_targets, blocks, part_doubles, &chunk)
             : direct_splits(n, n_targets, blocks, n_targets * 3, &chunk);
    const size_t tblocks = (n_targets + kDirThreads * kDirPer - 1) / (kDirThreads * kDirPer);
    dim3 grid((unsigned)tblocks, (unsigned)splits);
    if (splits == 1) {
        k_direct_f64<<<grid, kDirThreads, 0, st>>>(xyzm, n, targets, n_targets, chunk, out);
        return;
    }
    k_direct_f64<<<grid, kDirThreads, 0, st>>>(xyzm, n, targets, n_targets, chunk, part);
    const size_t m = n_targets * 3;
    const unsigned g = (unsigned)((m + 255) / 256 < 1024 ? (m + 255) / 256 : 1024);
    k_direct_sum<<<g, 256, 0, st>>>(part, m, (int)splits, out);
}

}  // namespace psg
