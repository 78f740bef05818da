// Octree build from the sorted Morton codes, and the upward pass (P2M/M2M).
//
// Reference: ps_impl_build_tree (polesitter.h:906-967) recursively splits a
// node [s, e) at depth d < 10 holding >= 2 particles into one child per
// non-empty octant of digit (code >> (27 - 3d)) & 7; a node is a leaf when
// d == 10 or it holds <= 1 particle (:911-916).  Equivalently, with
// cpl(i) = the number of leading octal digits codes[i-1] and codes[i] share,
// a depth-d node starts at position i iff
//     (i == 0 or cpl(i) < d)                        -- a depth-d run starts
// and (cpl(i) >= d-1 or cpl(i+1) >= d-1)            -- its parent run has >= 2
// so the whole tree comes from one pass of flags and a 10-wide prefix scan,
// with no recursion.  Levels are stored contiguously in Morton order.
//
// Leaf capacity B > 1 (an extension: nodes holding <= B particles are
// leaves): "its parent run has >= 2" becomes "> B".  The depth-k runs
// around i shrink as k grows, and the depth-k run holding i has > B
// particles iff some window [j, j+B] containing i lies inside it, so a
// depth-d node starts at i iff a depth-d run starts there and
//     d - 1 <= W(i) = max over j in [i-B, i] of cpl2(codes[j], codes[j+B])
// (cpl2 = common octal prefix length).  With B = 1 this is the rule above.
// The root is split whenever it holds >= 2 particles, so every particle has
// a leaf below the root (W(i) >= 0).
//
// Child centres follow the reference's float chain exactly (:935-939):
// hw_child = hw * 0.5 and c_child = c_parent +/- hw_child, replayed from the
// root for each node.
#include "psg_common.cuh"
#include "psg_kernels.h"

namespace psg {

constexpr int kTreeThreads = 256;
constexpr int kTreePer = 4;
constexpr int kTreeTile = kTreeThreads * kTreePer;  // 1024 positions

int tree_tile_size() { return kTreeTile; }

__device__ __forceinline__ int cpl2(uint32_t a, uint32_t b) {
    // common octal prefix length of two codes (0 .. 10)
    const uint32_t x = (a ^ b) & 0x3FFFFFFFu;
    if (x == 0u) return kMaxDepth;
    return (__clz(x) - 2) / 3;
}

__device__ __forceinline__ int cpl_at(const uint32_t* __restrict__ c, size_t i, size_t n) {
    // common octal prefix length of codes[i-1], codes[i]; -1 outside [1, n)
    if (i == 0 || i >= n) return -1;
    return cpl2(c[i - 1], c[i]);
}

// 10 one-bit flags (bit d-1 <=> a depth-d node starts at i); w = W(i), the
// deepest level whose run around i holds more than the leaf capacity
__device__ __forceinline__ uint32_t node_flags(int cpl_i, int w, bool first) {
    uint32_t f = 0;
#pragma unroll
    for (int d = 1; d <= kMaxDepth; ++d) {
        bool start = first || cpl_i < d;
        if (start && w >= d - 1) f |= 1u << (d - 1);
    }
    return f;
}

// counters of depths 1..5 in lo, 6..10 in hi, 12 bits each
__device__ __forceinline__ void add_flags(unsigned long long& lo, unsigned long long& hi,
                                          uint32_t f) {
#pragma unroll
    for (int d = 0; d < 5; ++d) {
        lo += (unsigned long long)((f >> d) & 1u) << (12 * d);
        hi += (unsigned long long)((f >> (d + 5)) & 1u) << (12 * d);
    }
}

__device__ __forceinline__ uint32_t get_cnt(unsigned long long lo, unsigned long long hi,
                                            int d /*1..10*/) {
    return d <= 5 ? (uint32_t)((lo >> (12 * (d - 1))) & 0xFFFull)
                  : (uint32_t)((hi >> (12 * (d - 6))) & 0xFFFull);
}

__device__ __forceinline__ void thread_flags(const uint32_t* __restrict__ codes, size_t n,
                                             size_t p0, uint32_t cap,
                                             uint32_t (&f)[kTreePer]) {
    int cprev = cpl_at(codes, p0, n);
    if (cap <= 1u) {
        // W(i) = max(cpl(i), cpl(i+1))
#pragma unroll
        for (int q = 0; q < kTreePer; ++q) {
            size_t i = p0 + q;
            int cnext = cpl_at(codes, i + 1, n);
            f[q] = (i < n) ? node_flags(cprev, max(cprev, cnext), i == 0) : 0u;
            cprev = cnext;
        }
        return;
    }
    // W over the windows [j, j + cap] with j in [p0 - cap, p0 + kTreePer - 1],
    // 0 <= j and j + cap < n; at least 0 (the root is split) once n >= 2
    int w[kTreePer];
#pragma unroll
    for (int q = 0; q < kTreePer; ++q) w[q] = n >= 2 ? 0 : -1;
    const long long jlo = max(0ll, (long long)p0 - (long long)cap);
    const long long jhi = min((long long)p0 + kTreePer - 1, (long long)n - 1 - (long long)cap);
#pragma unroll 4
    for (long long j = jlo; j <= jhi; ++j) {
        const int c = cpl2(codes[j], codes[j + cap]);
#pragma unroll
        for (int q = 0; q < kTreePer; ++q) {
            const long long i = (long long)p0 + q;
            if (j <= i && j + (long long)cap >= i) w[q] = max(w[q], c);
        }
    }
#pragma unroll
    for (int q = 0; q < kTreePer; ++q) {
        size_t i = p0 + q;
        f[q] = (i < n) ? node_flags(cprev, w[q], i == 0) : 0u;
        cprev = cpl_at(codes, i + 1, n);
    }
}

// Many systems in one array: the same rules inside each system's range,
// with its own leaf capacity; a system's first position starts its root (a
// depth-0 node, node k of level 0) and no run crosses a system boundary.
__device__ __forceinline__ void thread_flags_forest(const uint32_t* __restrict__ codes, size_t n,
                                                    size_t p0, const TreeView& tv,
                                                    uint32_t (&f)[kTreePer]) {
#pragma unroll 1
    for (int q = 0; q < kTreePer; ++q) {
        const size_t i = p0 + q;
        if (i >= n) {
            f[q] = 0u;
            continue;
        }
        const uint32_t k = tv.part_sys[i];
        const size_t lo = tv.sys_off[k], hi = tv.sys_off[k + 1];
        const uint32_t cap = tv.sys_cap[k];
        const bool first = i == lo;
        const int cpl_i = first ? -1 : cpl2(codes[i - 1], codes[i]);
        int w;
        if (cap <= 1u) {
            const int cnext = i + 1 < hi ? cpl2(codes[i], codes[i + 1]) : -1;
            w = max(cpl_i, cnext);
        } else {
            w = hi - lo >= 2 ? 0 : -1;
            const size_t jlo = i >= lo + cap ? i - cap : lo;
            if (hi >= lo + cap + 1) {
                const size_t jhi = min(i, hi - 1 - cap);
                for (size_t j = jlo; j <= jhi; ++j) w = max(w, cpl2(codes[j], codes[j + cap]));
            }
        }
        f[q] = node_flags(cpl_i, w, first);
    }
}

__global__ void __launch_bounds__(kTreeThreads) k_tree_count(const uint32_t* __restrict__ codes,
                                                            size_t n, uint32_t cap,
                                                            uint32_t* __restrict__ tile_cnt,
                                                            const TreeView tv) {
    const size_t p0 = (size_t)blockIdx.x * kTreeTile + (size_t)threadIdx.x * kTreePer;
    uint32_t f[kTreePer];
    if (tv.part_sys) thread_flags_forest(codes, n, p0, tv, f);
    else thread_flags(codes, n, p0, cap, f);
    unsigned long long lo = 0, hi = 0;
#pragma unroll
    for (int q = 0; q < kTreePer; ++q) add_flags(lo, hi, f[q]);
    lo = warp_sum(lo);
    hi = warp_sum(hi);
    __shared__ unsigned long long s[2][kTreeThreads / 32];
    if (lane_id() == 0) {
        s[0][threadIdx.x >> 5] = lo;
        s[1][threadIdx.x >> 5] = hi;
    }
    __syncthreads();
    if (threadIdx.x < kMaxDepth) {
        const int d = threadIdx.x + 1;
        uint32_t c = 0;
        for (int w = 0; w < kTreeThreads / 32; ++w) c += get_cnt(s[0][w], s[1][w], d);
        tile_cnt[(size_t)blockIdx.x * kMaxDepth + threadIdx.x] = c;
    }
}

// Exclusive scan of the tile counts per depth (one block of 1024 threads).
__global__ void __launch_bounds__(1024) k_tree_scan(uint32_t* __restrict__ tile_cnt, int tiles,
                                                    TreeView tv, Status* status) {
    __shared__ uint32_t wsum[32];
    __shared__ uint32_t carry;
    for (int d = 1; d <= kMaxDepth; ++d) {
        if (threadIdx.x == 0) carry = 0;
        __syncthreads();
        for (int b0 = 0; b0 < tiles; b0 += 1024) {
            int b = b0 + threadIdx.x;
            uint32_t v = b < tiles ? tile_cnt[(size_t)b * kMaxDepth + d - 1] : 0u;
            uint32_t inc = warp_incl_scan(v);
            if (lane_id() == 31) wsum[threadIdx.x >> 5] = inc;
            __syncthreads();
            uint32_t add = carry;
            for (int w = 0; w < (int)(threadIdx.x >> 5); ++w) add += wsum[w];
            if (b < tiles) tile_cnt[(size_t)b * kMaxDepth + d - 1] = inc - v + add;
            __syncthreads();
            if (threadIdx.x == 1023) carry = add + inc;
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            uint32_t total = carry;
            if (total > tv.lvl_cap[d]) {
                set_err(status, PSG_ERR_NODES);
                total = tv.lvl_cap[d];
            }
            status->lvl_count[d] = total;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        status->lvl_count[0] = tv.part_sys ? tv.nsys : 1u;
        status->lvl_count[kLevels] = 0;
    }
}

// centre of the node whose first code is `code` at depth d: the reference's
// chain of d rounded adds from the root centre
__device__ __forceinline__ float4 node_centre(uint32_t code, int d, float cx, float cy, float cz,
                                              float hw) {
    for (int l = 1; l <= d; ++l) {
        hw = __fmul_rn(hw, 0.5f);
        uint32_t dig = (code >> (30 - 3 * l)) & 7u;
        cx = __fadd_rn(cx, (dig & 1u) ? hw : -hw);
        cy = __fadd_rn(cy, (dig & 2u) ? hw : -hw);
        cz = __fadd_rn(cz, (dig & 4u) ? hw : -hw);
    }
    return make_float4(cx, cy, cz, hw);
}

// end of the run of codes sharing code[i]'s first d octal digits (gallop,
// then binary search)
__device__ __forceinline__ size_t run_end(const uint32_t* __restrict__ c, size_t n, size_t i,
                                          int d) {
    const int sh = 30 - 3 * d;
    const uint32_t key = (c[i] & 0x3FFFFFFFu) >> sh;
    size_t lo = i, step = 1;  // invariant: prefix(c[lo]) == key
    while (lo + step < n && ((c[lo + step] & 0x3FFFFFFFu) >> sh) == key) {
        lo += step;
        step <<= 1;
    }
    size_t hi = (lo + step < n) ? lo + step : n;  // prefix(c[hi]) != key or hi == n
    while (hi - lo > 1) {
        size_t mid = lo + ((hi - lo) >> 1);
        if (((c[mid] & 0x3FFFFFFFu) >> sh) == key) lo = mid; else hi = mid;
    }
    return hi;
}

__global__ void __launch_bounds__(kTreeThreads) k_tree_emit(const uint32_t* __restrict__ codes,
                                                           size_t n,
                                                           const uint32_t* __restrict__ tile_off,
                                                           TreeView tv, const Status* status,
                                                           float cx, float cy, float cz,
                                                           float hw,
                                                           const float* __restrict__ bbox,
                                                           uint32_t cap) {
    if (bbox) {
        // root from a device-side bounding box (min, max, range), as the
        // caller's loop derives it: c = min + range / 2, hw = range / 2
        // (README.md:76-78)
        hw = __fdiv_rn(bbox[2], 2.0f);
        cx = cy = cz = __fadd_rn(bbox[0], hw);
    }
    const size_t p0 = (size_t)blockIdx.x * kTreeTile + (size_t)threadIdx.x * kTreePer;
    uint32_t f[kTreePer];
    const bool forest = tv.part_sys != nullptr;
    if (forest) thread_flags_forest(codes, n, p0, tv, f);
    else thread_flags(codes, n, p0, cap, f);
    unsigned long long lo = 0, hi = 0;
#pragma unroll
    for (int q = 0; q < kTreePer; ++q) add_flags(lo, hi, f[q]);
    // block exclusive scan of the packed counters
    unsigned long long ilo = lo, ihi = hi;
    const uint32_t l = lane_id(), w = threadIdx.x >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        unsigned long long a = __shfl_up_sync(0xFFFFFFFFu, ilo, o);
        unsigned long long b = __shfl_up_sync(0xFFFFFFFFu, ihi, o);
        if (l >= (uint32_t)o) {
            ilo += a;
            ihi += b;
        }
    }
    __shared__ unsigned long long s[2][kTreeThreads / 32];
    __shared__ uint32_t s_off[kMaxDepth + 1];
    if (l == 31) {
        s[0][w] = ilo;
        s[1][w] = ihi;
    }
    if (threadIdx.x < kMaxDepth)
        s_off[threadIdx.x + 1] = tile_off[(size_t)blockIdx.x * kMaxDepth + threadIdx.x];
    __syncthreads();
    unsigned long long elo = ilo - lo, ehi = ihi - hi;
    for (uint32_t j = 0; j < w; ++j) {
        elo += s[0][j];
        ehi += s[1][j];
    }
    uint32_t rank[kMaxDepth + 2];
#pragma unroll
    for (int d = 1; d <= kMaxDepth; ++d)
        rank[d] = tv.lvl_base[d] + s_off[d] + get_cnt(elo, ehi, d);
    rank[kMaxDepth + 1] = 0;

    if (p0 == 0 && !forest) {  // root
        tv.geo[0] = make_float4(cx, cy, cz, hw);
        tv.info[0] = make_uint4(0u, (uint32_t)n, tv.lvl_base[1], pack_flags(0, 0, 0));
        tv.parent[0] = kNone;
        tv.cbase[0] = tv.lvl_base[1];
        tv.arrive[0] = 0;
        tv.lt[0] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
#pragma unroll
    for (int q = 0; q < kTreePer; ++q) {
        const size_t i = p0 + q;
        const uint32_t fq = f[q];
        uint32_t sys = 0;
        if (forest && i < n) {
            // this position's system: its root box (README.md:76-78) and, at
            // its first position, its root node
            sys = tv.part_sys[i];
            const float* bb = tv.sys_bbox + 4 * sys;
            hw = __fdiv_rn(bb[2], 2.0f);
            cx = cy = cz = __fadd_rn(bb[0], hw);
            const uint32_t lo_s = tv.sys_off[sys];
            if (i == lo_s) {
                tv.geo[sys] = make_float4(cx, cy, cz, hw);
                tv.info[sys] = make_uint4(lo_s, tv.sys_off[sys + 1] - lo_s, rank[1],
                                          pack_flags(0, 0, 0));
                tv.parent[sys] = kNone;
                tv.cbase[sys] = rank[1];
                tv.arrive[sys] = 0;
                tv.lt[sys] = make_float4(0.f, 0.f, 0.f, 0.f);
            }
        }
        if (fq) {
            const uint32_t code = codes[i];
            const size_t run_n = forest ? tv.sys_off[sys + 1] : n;
#pragma unroll 1
            for (int d = 1; d <= kMaxDepth; ++d) {
                if (!((fq >> (d - 1)) & 1u)) continue;
                const uint32_t id = rank[d];
                if (id - tv.lvl_base[d] >= status->lvl_count[d]) continue;  // capacity guard
                const size_t end = run_end(codes, run_n, i, d);
                const uint32_t cnt = (uint32_t)(end - i);
                uint32_t par = forest ? sys : 0u;
                if (d > 1) par = rank[d - 1] + ((fq >> (d - 2)) & 1u) - 1u;
                const uint32_t cb = d < kMaxDepth ? rank[d + 1] : 0u;
                tv.geo[id] = node_centre(code, d, cx, cy, cz, hw);
                tv.info[id] = make_uint4((uint32_t)i, cnt, cb,
                                         pack_flags(0, d, (code >> (30 - 3 * d)) & 7u));
                tv.parent[id] = par;
                tv.cbase[id] = cb;
                tv.arrive[id] = 0;
            }
        }
#pragma unroll
        for (int d = 1; d <= kMaxDepth; ++d) rank[d] += (fq >> (d - 1)) & 1u;
    }
}

// child count = next node's first-child rank - this node's (same level);
// also the particle count of the fullest leaf
__global__ void __launch_bounds__(256) k_tree_link(TreeView tv, const Status* status) {
    const uint32_t total = tv.lvl_base[kLevels];
    const uint32_t stride = gridDim.x * blockDim.x;
    uint32_t max_leaf = 0;
    for (uint32_t id = blockIdx.x * blockDim.x + threadIdx.x; id < total; id += stride) {
        int d = 0;
        while (d < kMaxDepth && id >= tv.lvl_base[d + 1]) ++d;
        const uint32_t r = id - tv.lvl_base[d];
        const uint32_t cnt_d = status->lvl_count[d];
        if (r >= cnt_d) continue;
        uint32_t nch = 0;
        if (d < kMaxDepth) {
            const uint32_t next = (r + 1 < cnt_d) ? tv.cbase[id + 1]
                                                  : tv.lvl_base[d + 1] + status->lvl_count[d + 1];
            nch = next - tv.cbase[id];
            if (nch > 8u) {  // codes not sorted by their 30-bit prefix
                set_err(const_cast<Status*>(status), PSG_ERR_NODES);
                nch = 0;
            }
        }
        uint4 inf = tv.info[id];
        inf.w = (inf.w & ~0xFu) | (nch & 0xFu);
        tv.info[id] = inf;
        tv.link[id] = nch ? ((inf.z & kLinkMask) | (nch << 28)) : 0u;
        tv.lt[id] = make_float4(0.f, 0.f, 0.f, 0.f);
        if (nch == 0 && inf.y > max_leaf) max_leaf = inf.y;
        // batched systems: each system picks its own leaf-pass variant
        if (nch == 0 && tv.part_sys && inf.y >= 32u)
            atomicMax(&tv.sys_maxleaf[tv.part_sys[inf.x]], inf.y);
    }
    max_leaf = __reduce_max_sync(0xFFFFFFFFu, max_leaf);
    if (lane_id() == 0 && max_leaf) atomicMax(&const_cast<Status*>(status)->max_leaf, max_leaf);
}

// Upward pass, one launch per level from the deepest up: a leaf sums P2M
// over its particles, an internal node adds its children's multipoles (M2M).
// Operation order matches polesitter.h:978-1045 exactly (sequential sums over
// the leaf's particles; children in octant order), every op rounded to nearest.
__global__ void __launch_bounds__(256) k_upward_level(TreeView tv, const Status* status,
                                                      const float4* __restrict__ xyzm, int d) {
    if (status->err & (PSG_ERR_NODES | PSG_ERR_SORT_SPIN)) return;
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= status->lvl_count[d]) return;
    const uint32_t id = tv.lvl_base[d] + r;
    const float4 c = tv.geo[id];
    const uint32_t link = tv.link[id];
    float m0 = 0.f, mx = 0.f, my = 0.f, mz = 0.f;
    if ((link >> 28) == 0) {
        const uint4 inf = tv.info[id];
        for (uint32_t k = 0; k < inf.y; ++k) {
            const float4 p = xyzm[inf.x + k];
            m0 = __fadd_rn(m0, p.w);
            mx = __fadd_rn(mx, __fmul_rn(p.w, __fsub_rn(p.x, c.x)));
            my = __fadd_rn(my, __fmul_rn(p.w, __fsub_rn(p.y, c.y)));
            mz = __fadd_rn(mz, __fmul_rn(p.w, __fsub_rn(p.z, c.z)));
        }
    } else {
        const uint32_t fc = link & kLinkMask, nch = link >> 28;
        for (uint32_t j = 0; j < nch; ++j) {
            const float4 cm = tv.mp[fc + j];
            const float4 cg = tv.geo[fc + j];
            m0 = __fadd_rn(m0, cm.x);
            mx = __fadd_rn(mx, __fadd_rn(cm.y, __fmul_rn(cm.x, __fsub_rn(cg.x, c.x))));
            my = __fadd_rn(my, __fadd_rn(cm.z, __fmul_rn(cm.x, __fsub_rn(cg.y, c.y))));
            mz = __fadd_rn(mz, __fadd_rn(cm.w, __fmul_rn(cm.x, __fsub_rn(cg.z, c.z))));
        }
    }
    tv.mp[id] = make_float4(m0, mx, my, mz);
}

void launch_tree(const uint32_t* codes, size_t n, uint32_t* tile_buf, TreeView tv,
                 Status* status, float cx, float cy, float cz, float hw, int grid,
                 cudaStream_t st, const float* bbox, uint32_t leaf_cap) {
    const int tiles = (int)((n + kTreeTile - 1) / kTreeTile);
    k_tree_count<<<tiles, kTreeThreads, 0, st>>>(codes, n, leaf_cap, tile_buf, tv);
    k_tree_scan<<<1, 1024, 0, st>>>(tile_buf, tiles, tv, status);
    k_tree_emit<<<tiles, kTreeThreads, 0, st>>>(codes, n, tile_buf, tv, status, cx, cy, cz, hw,
                                                bbox, leaf_cap);
    k_tree_link<<<grid, 256, 0, st>>>(tv, status);
}

void launch_upward(TreeView tv, const Status* status, const float4* xyzm, int grid,
                   cudaStream_t st) {
    (void)grid;
    for (int d = kMaxDepth; d >= 0; --d) {
        const int g = (int)((tv.lvl_cap[d] + 255) / 256);
        k_upward_level<<<g, 256, 0, st>>>(tv, status, xyzm, d);
    }
}

}  // namespace psg
