// Stable LSD radix sort of the Morton codes with the particle index as
// payload, then one gather of (x, y, z, mass) and ids into sorted order.
//
// Reference: ps_impl_sort_particles (polesitter.h:1588-1693) sorts the six
// arrays with four stable 8-bit LSD passes on the CPU.  Any stable sort by
// the full 32-bit code yields the same permutation; here each pass is one
// "onesweep" kernel: a tile ranks its keys per warp with match_any, takes its
// global digit offsets from the tiles before it by decoupled look-back (every
// wait is bounded; a timeout raises PSG_ERR_SORT_SPIN instead of hanging),
// and scatters through shared memory so each digit run is written
// contiguously.  Traffic per pass: 8 B read + 8 B written per key.
#include "psg_common.cuh"
#include "psg_kernels.h"

namespace psg {

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortItems = 8;
constexpr int kSortTile = kSortThreads * kSortItems;  // 2048 keys
constexpr uint32_t kFlagAgg = 1u << 30;
constexpr uint32_t kFlagInc = 2u << 30;
constexpr uint32_t kValMask = (1u << 30) - 1;
constexpr int kSpinLimit = 1 << 22;
constexpr unsigned long long kLateNs = 200000;  // the late tile of the wait test: 200 us

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

int sort_tile_size() { return kSortTile; }

// Histograms of all four digits in one read of the keys.
__global__ void __launch_bounds__(256) k_sort_hist(const uint32_t* __restrict__ keys, size_t n,
                                                   uint32_t* __restrict__ hist /*[4][256]*/) {
    __shared__ uint32_t h[4][256];
    for (int i = threadIdx.x; i < 1024; i += blockDim.x) (&h[0][0])[i] = 0;
    __syncthreads();
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        uint32_t k = __ldg(keys + i);
        atomicAdd(&h[0][k & 0xFFu], 1u);
        atomicAdd(&h[1][(k >> 8) & 0xFFu], 1u);
        atomicAdd(&h[2][(k >> 16) & 0xFFu], 1u);
        atomicAdd(&h[3][k >> 24], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 1024; i += blockDim.x) {
        uint32_t v = (&h[0][0])[i];
        if (v) atomicAdd(hist + i, v);
    }
}

// Exclusive scan of each pass's 256 digit counts (one block of 256 threads).
__global__ void __launch_bounds__(256) k_sort_scan(const uint32_t* __restrict__ hist,
                                                   uint32_t* __restrict__ offs) {
    __shared__ uint32_t wsum[8];
    const int t = threadIdx.x, w = t >> 5;
    for (int p = 0; p < 4; ++p) {
        uint32_t v = hist[p * 256 + t];
        uint32_t inc = warp_incl_scan(v);
        if ((t & 31) == 31) wsum[w] = inc;
        __syncthreads();
        uint32_t add = 0;
        for (int j = 0; j < w; ++j) add += wsum[j];
        offs[p * 256 + t] = inc - v + add;
        __syncthreads();
    }
}

// One stable pass on the 8-bit digit (key >> shift) & 0xFF; offs: the
// pass's 256 global digit starts.
__global__ void __launch_bounds__(kSortThreads) k_sort_pass(
    const uint32_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in,
    uint32_t* __restrict__ keys_out, uint32_t* __restrict__ vals_out, size_t n, int shift,
    const uint32_t* __restrict__ offs /*[256]*/, uint32_t* lookback /*[tiles][256]*/,
    uint32_t* ticket, Status* status, int spin_limit, int late) {
    __shared__ uint32_t s_wcnt[kSortWarps][256];
    __shared__ uint32_t s_keys[kSortTile];
    __shared__ uint32_t s_vals[kSortTile];
    __shared__ uint32_t s_dstart[256];
    __shared__ uint32_t s_glob[256];
    __shared__ uint32_t s_wsum[kSortWarps];
    __shared__ uint32_t s_tile;

    const int t = threadIdx.x, w = t >> 5, l = t & 31;
    if (t == 0) s_tile = atomicAdd(ticket, 1u);
    for (int i = t; i < kSortWarps * 256; i += kSortThreads) (&s_wcnt[0][0])[i] = 0;
    __syncthreads();
    const uint32_t tile = s_tile;
    const size_t base = (size_t)tile * kSortTile;

    uint32_t key[kSortItems], val[kSortItems], rank[kSortItems];
#pragma unroll
    for (int it = 0; it < kSortItems; ++it) {
        size_t idx = base + (size_t)w * 32 * kSortItems + (size_t)it * 32 + l;
        if (idx < n) {
            key[it] = keys_in[idx];
            val[it] = vals_in ? vals_in[idx] : (uint32_t)idx;
        } else {
            key[it] = 0;
            val[it] = 0;
        }
    }
    // Per-warp stable ranking: items are visited in index order (item-major,
    // lane-minor), so equal digits keep their input order.
    const uint32_t lt = lanemask_lt();
#pragma unroll
    for (int it = 0; it < kSortItems; ++it) {
        const bool valid = (base + (size_t)w * 32 * kSortItems + (size_t)it * 32 + l) < n;
        uint32_t d = valid ? ((key[it] >> shift) & 0xFFu) : 256u;
        uint32_t peers = __match_any_sync(0xFFFFFFFFu, d);
        uint32_t before = (d < 256u) ? s_wcnt[w][d] : 0u;
        rank[it] = before + __popc(peers & lt);
        __syncwarp();
        if (d < 256u && (__ffs(peers) - 1) == l) s_wcnt[w][d] = before + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    // thread t owns digit t: exclusive prefix over warps, tile total
    uint32_t total = 0;
#pragma unroll
    for (int j = 0; j < kSortWarps; ++j) {
        uint32_t c = s_wcnt[j][t];
        s_wcnt[j][t] = total;
        total += c;
    }
    // publish this tile's aggregate, then look back for the exclusive prefix
    uint32_t* my = lookback + (size_t)tile * 256 + t;
    uint32_t prefix = 0;
    if (tile == 0) {
        if (late) {
            // test of the bounded wait: this tile publishes ~200 us late, so
            // a successor polling fewer times gives up (bounded: at most
            // 2^20 reads of the clock)
            const unsigned long long t0 = global_ns();
            for (int i = 0; i < (1 << 20) && global_ns() - t0 < kLateNs; ++i) {
            }
        }
        atomicExch(my, kFlagInc | total);
    } else {
        atomicExch(my, kFlagAgg | total);
        int j = (int)tile - 1;
        int spins = 0;
        while (j >= 0) {
            uint32_t v = *((volatile uint32_t*)(lookback + (size_t)j * 256 + t));
            uint32_t f = v & ~kValMask;
            if (f == 0u) {
                if (++spins > spin_limit) {
                    set_err(status, PSG_ERR_SORT_SPIN);
                    break;
                }
                continue;
            }
            prefix += v & kValMask;
            if (f == kFlagInc) break;
            --j;
        }
        atomicExch(my, kFlagInc | (prefix + total));
    }
    s_glob[t] = offs[t] + prefix;
    // tile-local digit starts: exclusive scan of totals over digits
    uint32_t inc = warp_incl_scan(total);
    if (l == 31) s_wsum[w] = inc;
    __syncthreads();
    uint32_t add = 0;
    for (int j = 0; j < w; ++j) add += s_wsum[j];
    s_dstart[t] = inc - total + add;
    __syncthreads();
#pragma unroll
    for (int it = 0; it < kSortItems; ++it) {
        size_t idx = base + (size_t)w * 32 * kSortItems + (size_t)it * 32 + l;
        if (idx < n) {
            uint32_t d = (key[it] >> shift) & 0xFFu;
            uint32_t pos = s_dstart[d] + s_wcnt[w][d] + rank[it];
            s_keys[pos] = key[it];
            s_vals[pos] = val[it];
        }
    }
    __syncthreads();
    const uint32_t cnt = (uint32_t)((n - base) < (size_t)kSortTile ? (n - base) : kSortTile);
    for (uint32_t i = t; i < cnt; i += kSortThreads) {
        uint32_t k = s_keys[i];
        uint32_t d = (k >> shift) & 0xFFu;
        uint32_t dst = s_glob[d] + (i - s_dstart[d]);
        if (dst < n) {  // only false after a look-back timeout (error raised)
            keys_out[dst] = k;
            vals_out[dst] = s_vals[i];
        }
    }
}

// sorted (x, y, z, m) and ids: one random read of each source array
__global__ void __launch_bounds__(256) k_gather(const uint32_t* __restrict__ perm,
                                                const float* __restrict__ x,
                                                const float* __restrict__ y,
                                                const float* __restrict__ z,
                                                const float* __restrict__ m,
                                                const uint32_t* __restrict__ id, size_t n,
                                                float4* __restrict__ xyzm,
                                                uint32_t* __restrict__ ids) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += stride) {
        uint32_t i = perm[k];
        if (i >= n) i = 0;  // only after a sort error (raised in the status)
        xyzm[k] = make_float4(__ldg(x + i), __ldg(y + i), __ldg(z + i), __ldg(m + i));
        ids[k] = __ldg(id + i);
    }
}

// The reference leaves the caller's x, y, z, mass, id sorted in place
// (polesitter.h:1686-1690); write the sorted copies back.
__global__ void __launch_bounds__(256) k_writeback(const float4* __restrict__ xyzm,
                                                   const uint32_t* __restrict__ ids, size_t n,
                                                   float* __restrict__ x, float* __restrict__ y,
                                                   float* __restrict__ z, float* __restrict__ m,
                                                   uint32_t* __restrict__ id) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += stride) {
        float4 p = xyzm[k];
        x[k] = p.x;
        y[k] = p.y;
        z[k] = p.z;
        m[k] = p.w;
        id[k] = ids[k];
    }
}

void launch_sort(SortBuffers& b, uint32_t* codes, size_t n, int grid, Status* status,
                 cudaStream_t st, int spin_limit) {
    // spin_limit > 0: the wait test (that many polls; the first tile of the
    // first pass publishes late)
    const int limit = spin_limit > 0 ? spin_limit : kSpinLimit;
    const int tiles = (int)((n + kSortTile - 1) / kSortTile);
    cudaMemsetAsync(b.hist, 0, 4 * 256 * sizeof(uint32_t), st);
    cudaMemsetAsync(b.lookback, 0, (size_t)4 * tiles * 256 * sizeof(uint32_t), st);
    cudaMemsetAsync(status->sort_tiles, 0, sizeof(status->sort_tiles), st);
    k_sort_hist<<<grid, 256, 0, st>>>(codes, n, b.hist);
    k_sort_scan<<<1, 256, 0, st>>>(b.hist, b.offs);
    const uint32_t* kin = codes;
    const uint32_t* vin = nullptr;
    uint32_t* kouts[4] = {b.key_b, b.key_a, b.key_b, codes};
    uint32_t* vouts[4] = {b.val_b, b.val_a, b.val_b, b.val_a};
    for (int p = 0; p < 4; ++p) {
        k_sort_pass<<<tiles, kSortThreads, 0, st>>>(kin, vin, kouts[p], vouts[p], n, 8 * p,
                                                   b.offs + 256 * p,
                                                   b.lookback + (size_t)p * tiles * 256,
                                                   status->sort_tiles + p, status, limit,
                                                   spin_limit > 0 && p == 0 ? 1 : 0);
        kin = kouts[p];
        vin = vouts[p];
    }
    b.perm = b.val_a;
}

// the system of the particle at each position after the code passes
__global__ void __launch_bounds__(256) k_sort_sys_keys(const uint32_t* __restrict__ perm,
                                                       const uint32_t* __restrict__ part_sys,
                                                       size_t n, uint32_t* __restrict__ out) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint32_t j = perm[i];
        out[i] = j < n ? part_sys[j] : 0u;  // j >= n only after a sort error (raised)
    }
}

// codes in the final order, from the unsorted codes
__global__ void __launch_bounds__(256) k_sort_gather_codes(const uint32_t* __restrict__ perm,
                                                           const uint32_t* __restrict__ codes,
                                                           size_t n, uint32_t* __restrict__ out) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint32_t j = perm[i];
        out[i] = j < n ? codes[j] : 0u;
    }
}

// Many systems in one array, system k at [sys_off[k], sys_off[k+1]): every
// system's codes sorted stably within its own range, in one set of passes.
// The four code passes sort all particles by code; then stable passes on the
// system index (its low byte, then its high byte when there are more than
// 256 systems) put each system back in its range with its code order and
// ties kept -- the order each system's own sort gives.  The digit starts of
// the system passes come from the system sizes (sys_offs, host-computed,
// [passes][256]).
void launch_sort_forest(SortBuffers& b, uint32_t* codes, size_t n, int grid, Status* status,
                        cudaStream_t st, const uint32_t* part_sys, int sys_passes,
                        const uint32_t* sys_offs) {
    const int tiles = (int)((n + kSortTile - 1) / kSortTile);
    const int passes = 4 + sys_passes;
    cudaMemsetAsync(b.hist, 0, 4 * 256 * sizeof(uint32_t), st);
    cudaMemsetAsync(b.lookback, 0, (size_t)passes * tiles * 256 * sizeof(uint32_t), st);
    cudaMemsetAsync(status->sort_tiles, 0, sizeof(status->sort_tiles), st);
    k_sort_hist<<<grid, 256, 0, st>>>(codes, n, b.hist);
    k_sort_scan<<<1, 256, 0, st>>>(b.hist, b.offs);
    // code passes: codes -> b -> a -> b -> a (the input codes stay as they are)
    const uint32_t* kin = codes;
    const uint32_t* vin = nullptr;
    uint32_t* kouts[4] = {b.key_b, b.key_a, b.key_b, b.key_a};
    uint32_t* vouts[4] = {b.val_b, b.val_a, b.val_b, b.val_a};
    for (int p = 0; p < 4; ++p) {
        k_sort_pass<<<tiles, kSortThreads, 0, st>>>(kin, vin, kouts[p], vouts[p], n, 8 * p,
                                                   b.offs + 256 * p,
                                                   b.lookback + (size_t)p * tiles * 256,
                                                   status->sort_tiles + p, status, kSpinLimit,
                                                   0);
        kin = kouts[p];
        vin = vouts[p];
    }
    // system passes on (system index, permutation)
    k_sort_sys_keys<<<grid, 256, 0, st>>>(b.val_a, part_sys, n, b.key_b);
    uint32_t* sk[2] = {b.key_b, b.key_a};
    uint32_t* sv[2] = {b.val_a, b.val_b};
    for (int q = 0; q < sys_passes; ++q) {
        const int p = 4 + q;
        k_sort_pass<<<tiles, kSortThreads, 0, st>>>(sk[q & 1], sv[q & 1], sk[(q + 1) & 1],
                                                   sv[(q + 1) & 1], n, 8 * q,
                                                   sys_offs + 256 * q,
                                                   b.lookback + (size_t)p * tiles * 256,
                                                   status->sort_tiles + p, status, kSpinLimit,
                                                   0);
    }
    b.perm = sv[sys_passes & 1];
    // the codes in that order (key_b is free again: the system keys it held
    // were consumed, or it received the discarded keys of the last pass)
    k_sort_gather_codes<<<grid, 256, 0, st>>>(b.perm, codes, n, b.key_b);
    cudaMemcpyAsync(codes, b.key_b, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st);
}

void launch_gather(const uint32_t* perm, const float* x, const float* y, const float* z,
                   const float* m, const uint32_t* id, size_t n, float4* xyzm, uint32_t* ids,
                   int grid, cudaStream_t st) {
    k_gather<<<grid, 256, 0, st>>>(perm, x, y, z, m, id, n, xyzm, ids);
}

void launch_writeback(const float4* xyzm, const uint32_t* ids, size_t n, float* x, float* y,
                      float* z, float* m, uint32_t* id, int grid, cudaStream_t st) {
    k_writeback<<<grid, 256, 0, st>>>(xyzm, ids, n, x, y, z, m, id);
}

}  // namespace psg
