// Shared device-side definitions for the polesitter B200 FMM tick.
//
// Data layout in HBM (all arrays owned by one psg_ctx, sized from
// max_particles at ps_init):
//   particles, sorted: float4 xyzm[N] (x, y, z, mass), uint32 ids[N]
//   tree, level-major: level d occupies node ids [lvl_base[d],
//     lvl_base[d] + min(8^d, N)); inside a level nodes are in Morton order,
//     which is the order the reference's octant recursion creates them
//     (polesitter.h:923-966).  Per node:
//       float4 geo  (centre x, y, z, half_width)        polesitter.h:364-367
//       float4 mp   (m0, dipole x, y, z)                polesitter.h:370
//       float4 lt   (0, field x, y, z) = local_exp after the downward pass
//       uint4  info (first particle, count, first child, packed flags)
//       uint32 parent
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "psg_internal.h"

namespace psg {

constexpr int kMaxDepth = 10;   // PS_MAX_DEPTH, polesitter.h:882-883
constexpr int kLevels = kMaxDepth + 1;
constexpr uint32_t kNone = 0xFFFFFFFFu;
// node link word: first child id in the low 28 bits, child count (0..8,
// 0 = leaf) in the top 4
constexpr uint32_t kLinkMask = (1u << 28) - 1u;
// sources of a leaf's P2P list are stored in chained chunks of this size
constexpr int kP2PChunk = 32;

// info.w packing: nchild (4 bits) | depth << 4 (4 bits) | octant << 8 (3 bits)
__host__ __device__ inline uint32_t pack_flags(uint32_t nchild, uint32_t depth,
                                               uint32_t octant) {
    return nchild | (depth << 4) | (octant << 8);
}
__host__ __device__ inline uint32_t flags_nchild(uint32_t w) { return w & 0xFu; }
__host__ __device__ inline uint32_t flags_depth(uint32_t w) { return (w >> 4) & 0xFu; }
__host__ __device__ inline uint32_t flags_octant(uint32_t w) { return (w >> 8) & 0x7u; }

// Device view of the per-tick state, passed by value to kernels.
struct TreeView {
    float4* geo;
    float4* mp;
    float4* lt;
    uint4* info;
    uint32_t* parent;
    uint32_t* arrive;      // upward-pass arrival counters
    uint32_t* cbase;       // first-child rank per node (tree link step)
    uint32_t* link;        // first child | nchild << 28
    uint32_t* p2p_head;    // per leaf: last chunk of its P2P source list
    uint32_t* ns_off;      // per node: offset of its near-source list
    uint32_t* ns_cnt;      // per node: length of its near-source list
    uint32_t* dbg_m2l;     // per node M2L pair count (debug builds of a tick)
    uint32_t* dbg_p2p;     // per node P2P leaf-pair count (debug)
    float4* lg0;           // closure order 1: field gradient xx, yy, zz, xy
    float2* lg1;           //                  and xz, yz (null when unused)
    // many independent systems in one tree pass (the batched ensemble): the
    // particles of system k are [sys_off[k], sys_off[k + 1]), its root is
    // node k of level 0.  part_sys == null: one system, root node 0.
    const uint32_t* part_sys;   // system of each particle position
    const uint32_t* sys_off;    // [nsys + 1]
    const uint32_t* sys_cap;    // leaf capacity per system
    const float* sys_bbox;      // (min, max, range, 1023 / range) per system
    const float* sys_theta2;    // theta * theta (rounded) per system
    const int32_t* sys_heavy;   // shallow-leaf depth per system
    uint32_t* sys_maxleaf;      // particles in each system's fullest leaf (this tick)
    uint32_t nsys;
    uint32_t lvl_base[kLevels + 1];
    uint32_t lvl_cap[kLevels + 1];
};

// Device status block, copied to the host once at the end of a tick.
struct Status {
    uint32_t err;                          // PSG_ERR_* bits
    uint32_t lvl_count[kLevels + 1];       // nodes per level
    unsigned long long ns_used[kLevels + 1];  // near-list entries per level
    unsigned long long ns_cap;             // capacity of one near-list region
    uint32_t work[kLevels + 1];            // traversal work counters
    float bbox[4];                         // min, max, range, scale (prepare)
    unsigned long long stat[16];           // debug totals (see PSG_STAT_*)
    uint32_t max_stack;                    // deepest DFS stack seen (debug)
    uint32_t p2p_chunks;                   // P2P chunks used this tick
    uint32_t sort_tiles[6];                // onesweep tile tickets (code + system passes)
    uint32_t dense_count;                  // full-leaf P2P records written
    uint32_t dense_work;                   // ... and taken by k_dense_p2p
    uint32_t max_leaf;                     // particles in the fullest leaf
    uint32_t heavy_work;                   // groups taken by k_heavy_leaf
    uint32_t ns_fail;                      // bit k: level k's near lists did not fit
};

// P2P sources spilled from the traversal: chunk c holds cnt[c] source-leaf
// ids in src[c * kP2PChunk ...], each with the set of the group's children it
// serves in mask[...], and links to the group's previous chunk via next[c].
struct P2PStore {
    uint32_t* src;
    uint8_t* mask;
    uint32_t* next;
    uint32_t* cnt;
    uint32_t cap_chunks;
};

// The four float ops of the MAC, each rounded to nearest and never fused,
// in the reference's order (polesitter.h:1056-1064):
//   dist_sq = ((dx*dx) + (dy*dy)) + (dz*dz),  sep = dist_sq > (theta^2) * hw_sum^2
__device__ __forceinline__ bool mac_separated(float tx, float ty, float tz, float thw,
                                              float sx, float sy, float sz, float shw,
                                              float theta2, float& dx, float& dy,
                                              float& dz, float& d2) {
    dx = __fsub_rn(sx, tx);
    dy = __fsub_rn(sy, ty);
    dz = __fsub_rn(sz, tz);
    d2 = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
    float hs = __fadd_rn(thw, shw);
    return d2 > __fmul_rn(theta2, __fmul_rn(hs, hs));
}

__device__ __forceinline__ uint32_t lane_id() {
    uint32_t l;
    asm volatile("mov.u32 %0, %%laneid;" : "=r"(l));
    return l;
}

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm volatile("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    return v;
}

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v) {
    const uint32_t l = lane_id();
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xFFFFFFFFu, v, o);
        if (l >= (uint32_t)o) v += t;
    }
    return v;
}

__device__ __forceinline__ void set_err(Status* st, uint32_t bit) { atomicOr(&st->err, bit); }

}  // namespace psg
