// The interaction pass of the FMM tick: MAC + M2L + L2L, and for leaves also
// P2P + L2P, producing the final forces.
//
// Reference (PS_MULTITHREADING build): every node at depth 2, and every leaf
// above it, is paired with the root (ps_impl_dispatch_fmm, polesitter.h:
// 1772-1801, :1883-1885), and each pair (t, s) is walked by the dual
// recursion of ps_impl_fmm_interaction_pass (:1050-1146):
//   separated (MAC)        -> M2L: t.local += field of s's monopole+dipole
//   both leaves            -> P2P (the P2P pass :1258-1494 walks the same
//                             pairs with the same MAC)
//   t leaf                 -> (t, each child of s)
//   s leaf                 -> (each child of t, s)
//   otherwise              -> (each child of t) x (each child of s)
// then L2L adds every parent's field to its children (:1238-1251), L2P sets
// F = m * field at the leaves (:1224-1233) and P2P adds the direct sums
// f_t += m_t * sum_{j in s} m_j d / (|d|^2 + 0.1)^{3/2} (:1279-1449).
//
// B200 formulation (target-major, no interaction lists in HBM).  The pairs
// an internal target t hands to its children are its "near list" NS(t) =
// the sources it was not separated from, so all children of an internal
// node p (a "group") start from the same candidates
//   cand(p) = {root}                                         if depth(p) <= 1
//   cand(p) = U_{s in NS(p)} (s leaf ? {s} : children(s))    otherwise.
// One warp owns a group (with the closure's order-1 accumulators, half a
// group: children 0-3 or 4-7, so that the 4 x 9 accumulators leave room for
// 4 blocks per SM).  Candidates are tested 32 at a time, one per lane;
// each carries the set of the group's children it must be tested against,
// and the lane loads the candidate once and runs the MAC (and M2L, into
// per-child register accumulators) for each of those children.  What is
// not separated is dealt with once per chunk:
//
//  * MODE_INTERNAL, one launch per level k = 2..10, targets = the internal
//    children of the depth-(k-1) nodes: near candidates form NS(u) in HBM for
//    level k+1; L(u) = M2L(u) + L(p) is stored.
//  * MODE_LEAF, one launch after all levels, targets = the leaf children of
//    every node: a near leaf candidate is a P2P source, staged in shared
//    memory with the set of children it serves (spilled to HBM chunks past
//    128); a near internal candidate is the "t leaf" recursion -- it goes
//    onto a DFS stack in shared memory with the set of children that still
//    need it opened, so sibling leaves share every descent.  The warp then
//    finishes each leaf: L(u) = M2L(u) + L(p) and, per particle,
//    F = m * (L(u) + its P2P sum) -- written once, no atomics.  Running all
//    levels' leaves in one launch lets the long descents of shallow leaves
//    overlap with everything else.
//
// The MAC replays the reference's rounded float sequence exactly
// (mac_separated), so the interaction set is identical, ties included.
// Bound: FP32 pipe (M2L ~35 flop + 1 MUFU per pair; P2P ~20 flop + 1 MUFU
// per particle pair) and the latency of the candidate loads.
#include "psg_common.cuh"
#include "psg_kernels.h"

namespace psg {

constexpr int kTravWarps = 4;
constexpr int kTravThreads = kTravWarps * 32;
static_assert(kTravWarps == kDenseWarpsPerBlock, "k_dense_p2p runs kTravThreads a block");
constexpr int kCandBuf = 256;             // children of 32 opened entries
constexpr int kStackCap = 384;            // DFS stack (node, child mask)
constexpr int kStackSlack = 72;           // 9 levels x 7: growth of a single-entry descent
constexpr int kP2PCap = 128;              // staged P2P sources of a group
constexpr uint32_t kNsPool = 4096;        // near-list entries a warp reserves at once
constexpr uint32_t kChunkPool = 16;       // P2P spill chunks a warp reserves at once
constexpr uint32_t kDenseChunk = 32;      // target particles per dense work record
constexpr uint32_t kDenseSwitch = 32;     // fullest leaf from which the DENSE leaf pass runs
constexpr uint32_t kDenseCap = 8;         // ... or leaf capacity (leaves of many particles)

enum { MODE_INTERNAL = 0, MODE_LEAF = 1 };

struct SmemInternal {
    float4 cgeo[8];  // the group's children: centre + half width
    float4 cgp[4][2];  // ... pair-packed for the MAC (cgp_put)
    uint32_t cand_node[kCandBuf];
    uint32_t ns_cnt[8];
    uint32_t dbg_m2l[8];
    unsigned long long ns_next, ns_end;
    uint8_t cand_mask[kCandBuf];
};

struct SmemLeaf {
    float4 cgeo[8];
    float4 cgp[4][2];
    float4 chain_geo[8];    // chain groups: the ancestors a_{K+1} .. p under test
    float4 sL[8];           // the children's local fields
    float4 sG0[8];          // closure order 1: the children's field gradients
    float2 sG1[8];
    uint2 cpart[8];         // the children's particle ranges
    uint2 p2p_range[kP2PCap];
    uint32_t cand_node[kCandBuf];
    uint32_t stk_node[kStackCap];
    uint32_t p2p_node[kP2PCap];
    uint32_t chunk_next, chunk_end;
    uint32_t dbg_m2l[8];
    uint32_t dbg_p2p[8];
    uint8_t cand_mask[kCandBuf];
    uint8_t stk_mask[kStackCap];
    uint8_t p2p_mask[kP2PCap];
    uint8_t cand_lvl[kCandBuf];  // 0: tested against the children in the mask;
    uint8_t stk_lvl[kStackCap];  // c > 0: against chain target c (chain groups)
};

template <int MODE>
struct SmemOf { using T = SmemInternal; };
template <>
struct SmemOf<MODE_LEAF> { using T = SmemLeaf; };

__device__ __forceinline__ void m2l_field(float dx, float dy, float dz, float d2, float4 mp,
                                          float& fx, float& fy, float& fz) {
    // polesitter.h:1065-1092 with rsqrt: 1/r^3 and 1/r^5 of the softened distance
    const float soft = d2 + 0.1f;
    const float inv = rsqrtf(soft);
    const float inv2 = inv * inv;
    const float ir3 = inv2 * inv;
    const float ir5 = ir3 * inv2;
    const float mdr = fmaf(mp.y, dx, fmaf(mp.z, dy, mp.w * dz));
    const float a = fmaf(mp.x, ir3, -3.0f * mdr * ir5);
    fx = fmaf(dx, a, mp.y * ir3);
    fy = fmaf(dy, a, mp.z * ir3);
    fz = fmaf(dz, a, mp.w * ir3);
}

// m2l_field plus what the closure's order-1 local expansion needs: the
// gradient of the monopole field at the target centre is
// g3 * d d^T - gi * I with g3 = 3 m0 / r^5, gi = m0 / r^3 (softened r).
__device__ __forceinline__ void m2l_field_grad(float dx, float dy, float dz, float d2, float4 mp,
                                               float& fx, float& fy, float& fz, float& g3,
                                               float& gi) {
    const float soft = d2 + 0.1f;
    const float inv = rsqrtf(soft);
    const float inv2 = inv * inv;
    const float ir3 = inv2 * inv;
    const float ir5 = ir3 * inv2;
    const float mdr = fmaf(mp.y, dx, fmaf(mp.z, dy, mp.w * dz));
    const float a = fmaf(mp.x, ir3, -3.0f * mdr * ir5);
    fx = fmaf(dx, a, mp.y * ir3);
    fy = fmaf(dy, a, mp.z * ir3);
    fz = fmaf(dz, a, mp.w * ir3);
    g3 = 3.0f * mp.x * ir5;
    gi = mp.x * ir3;
}

// G v for the symmetric gradient stored as (xx, yy, zz, xy) + (xz, yz)
__device__ __forceinline__ float3 grad_apply(float4 g0, float2 g1, float vx, float vy, float vz) {
    return make_float3(fmaf(g0.x, vx, fmaf(g0.w, vy, g1.x * vz)),
                       fmaf(g0.w, vx, fmaf(g0.y, vy, g1.y * vz)),
                       fmaf(g1.x, vx, fmaf(g1.y, vy, g0.z * vz)));
}

// Children 2k and 2k + 1 of the group, pair-packed for the paired FP32
// instructions: cgp[k][0] = (x, x', y, y'), cgp[k][1] = (z, z', w, w');
// zeros past the nc children, so that every lane computes with finite
// values (a masked term is x * 0, which a NaN would survive).
// Warp-collective.
__device__ __forceinline__ void cgp_put(float4 (*cgp)[2], const float4* cgeo, uint32_t nc) {
    const uint32_t lane = lane_id();
    __syncwarp();
    if (lane < 4) {
        const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
        const float4 a = 2 * lane < nc ? cgeo[2 * lane] : z;
        const float4 b = 2 * lane + 1 < nc ? cgeo[2 * lane + 1] : z;
        cgp[lane][0] = make_float4(a.x, b.x, a.y, b.y);
        cgp[lane][1] = make_float4(a.z, b.z, a.w, b.w);
    }
    __syncwarp();
}

// Spill the group's staged P2P sources [0, fill) to HBM chunks of
// kP2PChunk (node, child mask) entries, chained to the group's earlier
// chunks.  Warp-collective; chunk ids come from a per-warp pool.  Returns the
// new chain head.
__device__ __noinline__ uint32_t spill_p2p(SmemLeaf& sm, uint32_t fill, uint32_t head,
                                           P2PStore st, Status* status) {
    const uint32_t lane = lane_id();
    for (uint32_t e0 = 0; e0 < fill; e0 += kP2PChunk) {
        if (sm.chunk_next >= sm.chunk_end) {
            uint32_t c = 0;
            if (lane == 0) c = atomicAdd(&status->p2p_chunks, kChunkPool);
            c = __shfl_sync(0xFFFFFFFFu, c, 0);
            __syncwarp();
            if (lane == 0) {
                sm.chunk_next = c;
                sm.chunk_end = c + kChunkPool;
            }
            __syncwarp();
        }
        const uint32_t c = sm.chunk_next;
        const uint32_t cnt = min((uint32_t)kP2PChunk, fill - e0);
        if (c < st.cap_chunks) {
            if (lane < cnt) {
                st.src[(size_t)c * kP2PChunk + lane] = sm.p2p_node[e0 + lane];
                st.mask[(size_t)c * kP2PChunk + lane] = sm.p2p_mask[e0 + lane];
            }
            if (lane == 0) {
                st.next[c] = head;
                st.cnt[c] = cnt;
            }
            head = c;
        } else if (lane == 0) {
            set_err(status, PSG_ERR_P2P_OVERFLOW);
        }
        __syncwarp();
        if (lane == 0) sm.chunk_next = c + 1;
        __syncwarp();
    }
    return head;
}

// Direct sum of the particles [r.x, r.x + r.y) on target particle t
// (polesitter.h:1424-1444 with rsqrt), optionally Kahan-compensated.
__device__ __forceinline__ void p2p_range(const float4* __restrict__ xyzm, uint2 r, float4 t,
                                          bool kahan, float& ax, float& ay, float& az, float& cx,
                                          float& cy, float& cz) {
    for (uint32_t j = 0; j < r.y; ++j) {
        const float4 p = xyzm[r.x + j];
        const float dx = p.x - t.x, dy = p.y - t.y, dz = p.z - t.z;
        const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz)) + 0.1f;
        const float inv = rsqrtf(r2);
        const float f = p.w * (inv * inv * inv);
        if (kahan) {
            const float yx = __fsub_rn(__fmul_rn(dx, f), cx);
            const float yy = __fsub_rn(__fmul_rn(dy, f), cy);
            const float yz = __fsub_rn(__fmul_rn(dz, f), cz);
            const float tx = __fadd_rn(ax, yx);
            const float ty = __fadd_rn(ay, yy);
            const float tz = __fadd_rn(az, yz);
            cx = __fsub_rn(__fsub_rn(tx, ax), yx);
            cy = __fsub_rn(__fsub_rn(ty, ay), yy);
            cz = __fsub_rn(__fsub_rn(tz, az), yz);
            ax = tx;
            ay = ty;
            az = tz;
        } else {
            ax = fmaf(dx, f, ax);
            ay = fmaf(dy, f, ay);
            az = fmaf(dz, f, az);
        }
    }
}

// k_dense_p2p work records for the leaf children in mask of the group whose
// children start at node fc: each run of consecutive children (their
// particles are contiguous) is cut into records of up to kDenseChunk
// particles; phead is the group's complete P2P source chain.
// Record: fc, phead, first particle, count | run's child mask << 8.
__device__ __noinline__ void record_dense(const SmemLeaf& sm, uint32_t mask, uint32_t fc,
                                          uint32_t phead, uint4* rec, uint32_t cap,
                                          Status* status) {
    const uint32_t lane = lane_id();
    while (mask) {
        const uint32_t q0 = __ffs(mask) - 1;
        uint32_t q1 = q0;
        while (q1 + 1 < 8 && ((mask >> (q1 + 1)) & 1u)) ++q1;
        const uint32_t run = ((2u << q1) - 1u) & ~((1u << q0) - 1u);
        mask &= ~run;
        const uint32_t first = sm.cpart[q0].x;
        uint32_t count = 0;
        for (uint32_t q = q0; q <= q1; ++q) count += sm.cpart[q].y;
        const uint32_t nrec = (count + kDenseChunk - 1) / kDenseChunk;
        uint32_t r0 = 0;
        if (lane == 0) r0 = atomicAdd(&status->dense_count, nrec);
        r0 = __shfl_sync(0xFFFFFFFFu, r0, 0);
        for (uint32_t k = lane; k < nrec; k += 32) {
            if (r0 + k < cap) {
                const uint32_t c0 = k * kDenseChunk;
                rec[r0 + k] = make_uint4(fc, phead, first + c0,
                                         min(kDenseChunk, count - c0) | (run << 8));
            }
        }
        if (lane == 0 && r0 + nrec > cap) set_err(status, PSG_ERR_DENSE_OVERFLOW);
    }
}

struct LeafOut {
    const float4* xyzm;
    const uint4* info;
    P2PStore p2p;
    float* fx;
    float* fy;
    float* fz;
    uint32_t* leaf_of;
    uint32_t* dbg_p2p;
    uint4* dense_rec;
    uint32_t dense_cap;
    int kahan;
};

// STREAM: the P2P sums of the staged sources [0, pfill) for every target
// particle of the work item's leaf children (tgt_mask), computed where they
// are found instead of spilled to HBM, so that no store grows with the size
// of a source list.  The children's particles are enumerated flat (children
// in mask order), 32 at a time; T lanes own targets (T the smallest power of
// two >= their count) and the 32 / T slices of lanes split the staged source
// leaves.  The slices' sums are added in a fixed order and kept in the force
// arrays between flushes (accum: add to what an earlier flush of this item
// left there).  fin: the item's last flush, which also applies L2P,
// F = m (L + all P2P sums), with order 1's shift to the particle.
template <bool DEBUG, bool GRAD>
__device__ __noinline__ void stream_p2p(SmemLeaf& sm, const LeafOut& o, uint32_t tgt_mask,
                                        uint32_t fc, uint32_t pfill, bool accum, bool fin,
                                        unsigned long long& inter) {
    const uint32_t lane = lane_id();
    for (uint32_t e = lane; e < pfill; e += 32) {
        const uint4 si = o.info[sm.p2p_node[e]];
        sm.p2p_range[e] = make_uint2(si.x, si.y);
    }
    __syncwarp();
    uint32_t total = 0;
    for (uint32_t m = tgt_mask; m; m &= m - 1) total += sm.cpart[__ffs(m) - 1].y;
    for (uint32_t r0 = 0; r0 < total; r0 += 32) {
        const uint32_t cnt = min(32u, total - r0);
        uint32_t T = 1;
        while (T < cnt) T <<= 1;
        const uint32_t S = 32u / T, tl = lane & (T - 1u), slice = lane / T;
        const bool active = tl < cnt;
        const uint32_t f = r0 + (active ? tl : 0u);
        uint32_t q = 0, i = 0, acc = 0;
        for (uint32_t m = tgt_mask; m; m &= m - 1) {
            const uint32_t qq = __ffs(m) - 1;
            const uint2 cp = sm.cpart[qq];
            if (f >= acc && f < acc + cp.y) {
                q = qq;
                i = cp.x + (f - acc);
            }
            acc += cp.y;
        }
        const float4 t = o.xyzm[i];
        float bx = 0.f, by = 0.f, bz = 0.f, cx = 0.f, cy = 0.f, cz = 0.f;
        uint32_t used = 0;
        for (uint32_t e = slice; e < pfill; e += S) {
            if ((sm.p2p_mask[e] >> q) & 1u) {
                const uint2 r = sm.p2p_range[e];
                p2p_range(o.xyzm, r, t, o.kahan, bx, by, bz, cx, cy, cz);
                used += r.y;
            }
        }
        bx -= cx;
        by -= cy;
        bz -= cz;
        for (uint32_t d = T; d < 32u; d <<= 1) {
            bx += __shfl_xor_sync(0xFFFFFFFFu, bx, d);
            by += __shfl_xor_sync(0xFFFFFFFFu, by, d);
            bz += __shfl_xor_sync(0xFFFFFFFFu, bz, d);
        }
        if (DEBUG) inter += active ? used : 0u;
        if (active && slice == 0) {
            if (accum) {
                bx += o.fx[i];
                by += o.fy[i];
                bz += o.fz[i];
            }
            if (!fin) {
                o.fx[i] = bx;
                o.fy[i] = by;
                o.fz[i] = bz;
            } else {
                const float4 L = sm.sL[q];
                float lx = L.y, ly = L.z, lz = L.w;
                if constexpr (GRAD) {
                    const float4 cu = sm.cgeo[q];
                    const float3 sh = grad_apply(sm.sG0[q], sm.sG1[q], t.x - cu.x, t.y - cu.y,
                                                 t.z - cu.z);
                    lx += sh.x;
                    ly += sh.y;
                    lz += sh.z;
                    if (o.leaf_of) o.leaf_of[i] = fc + q;
                }
                const double mm = (double)t.w;
                o.fx[i] = (float)(mm * ((double)lx + (double)bx));
                o.fy[i] = (float)(mm * ((double)ly + (double)by));
                o.fz[i] = (float)(mm * ((double)lz + (double)bz));
            }
        }
    }
    __syncwarp();
}

// L2P + P2P of a group's leaf children once its candidates are done: with
// DENSE, every group is handed to k_dense_p2p (which adds L and the P2P sum);
// otherwise F = m (L + P2P sum) here, one target particle at a time with the
// lanes over its sources.
template <bool DEBUG, bool GRAD, bool DENSE>
__device__ __forceinline__ void leaf_epilogue(SmemLeaf& sm, const LeafOut o, uint32_t tgt_mask,
                                           uint32_t fc, uint32_t pfill, uint32_t phead,
                                           bool stream, bool flushed,
                                           unsigned long long inter0, Status* status) {
    const uint32_t lane = lane_id();
    if (stream) {
        // the staged remainder, then L2P, in the warp (no spill, no records)
        unsigned long long inter = inter0;
        stream_p2p<DEBUG, GRAD>(sm, o, tgt_mask, fc, pfill, flushed, true, inter);
        if (DEBUG) {
            if (lane == 0) {
                for (uint32_t m = tgt_mask; m; m &= m - 1) {
                    const uint32_t q = __ffs(m) - 1;
                    o.dbg_p2p[fc + q] = sm.dbg_p2p[q];
                    atomicAdd(&status->stat[PSG_STAT_P2P_PAIRS],
                              (unsigned long long)sm.dbg_p2p[q]);
                }
            }
            inter = warp_sum(inter);
            if (lane == 0) atomicAdd(&status->stat[PSG_STAT_P2P_INTER], inter);
        }
        __syncwarp();
        return;
    }
    if constexpr (DENSE) {
        // the group's whole source list to HBM chunks, then k_dense_p2p work
        // records of up to 32 target particles
        if (pfill) phead = spill_p2p(sm, pfill, phead, o.p2p, status);
        record_dense(sm, tgt_mask, fc, phead, o.dense_rec, o.dense_cap, status);
        if (DEBUG && lane == 0) {
            for (uint32_t m = tgt_mask; m; m &= m - 1) {
                const uint32_t q = __ffs(m) - 1;
                o.dbg_p2p[fc + q] = sm.dbg_p2p[q];
                atomicAdd(&status->stat[PSG_STAT_P2P_PAIRS], (unsigned long long)sm.dbg_p2p[q]);
            }
        }
        __syncwarp();
        return;
    }
    // ---- L2P + P2P: F = m * (L(u) + sum of u's P2P sources) ----
    for (uint32_t e = lane; e < pfill; e += 32) {
        const uint4 si = o.info[sm.p2p_node[e]];
        sm.p2p_range[e] = make_uint2(si.x, si.y);
    }
    __syncwarp();
    unsigned long long inter = 0;
#pragma unroll 1
    for (uint32_t m = tgt_mask; m; m &= m - 1) {
        const uint32_t q = __ffs(m) - 1;
        const uint2 up = sm.cpart[q];
        const float4 L = sm.sL[q];
        for (uint32_t ti = 0; ti < up.y; ++ti) {
            const float4 t = o.xyzm[up.x + ti];
            float bx = 0.f, by = 0.f, bz = 0.f, cx = 0.f, cy = 0.f, cz = 0.f;
            for (uint32_t e = lane; e < pfill; e += 32) {
                if ((sm.p2p_mask[e] >> q) & 1u) {
                    const uint2 r = sm.p2p_range[e];
                    p2p_range(o.xyzm, r, t, o.kahan, bx, by, bz, cx, cy, cz);
                    if (DEBUG) inter += r.y;
                }
            }
            for (uint32_t c = phead; c != kNone; c = o.p2p.next[c]) {
                if (lane < o.p2p.cnt[c] &&
                    ((o.p2p.mask[(size_t)c * kP2PChunk + lane] >> q) & 1u)) {
                    const uint4 si = o.info[o.p2p.src[(size_t)c * kP2PChunk + lane]];
                    p2p_range(o.xyzm, make_uint2(si.x, si.y), t, o.kahan, bx, by, bz,
                              cx, cy, cz);
                    if (DEBUG) inter += si.y;
                }
            }
            const float sx = warp_sum(bx - cx);
            const float sy = warp_sum(by - cy);
            const float sz = warp_sum(bz - cz);
            if (lane == 0) {
                // final per-particle accumulation in FP64
                const size_t gi = (size_t)up.x + ti;
                const double mm = (double)t.w;
                float lx = L.y, ly = L.z, lz = L.w;
                if constexpr (GRAD) {
                    // order-1 L2P: the field at the particle
                    const float4 cu = sm.cgeo[q];
                    const float3 sh = grad_apply(sm.sG0[q], sm.sG1[q], t.x - cu.x,
                                                 t.y - cu.y, t.z - cu.z);
                    lx += sh.x;
                    ly += sh.y;
                    lz += sh.z;
                    if (o.leaf_of) o.leaf_of[gi] = fc + q;
                }
                o.fx[gi] = (float)(mm * ((double)lx + (double)sx));
                o.fy[gi] = (float)(mm * ((double)ly + (double)sy));
                o.fz[gi] = (float)(mm * ((double)lz + (double)sz));
            }
        }
        if (DEBUG && lane == 0) {
            o.dbg_p2p[fc + q] = sm.dbg_p2p[q];
            atomicAdd(&status->stat[PSG_STAT_P2P_PAIRS],
                      (unsigned long long)sm.dbg_p2p[q]);
        }
    }
    if (DEBUG) {
        inter = warp_sum(inter);
        if (lane == 0) atomicAdd(&status->stat[PSG_STAT_P2P_INTER], inter);
    }
    __syncwarp();
}

// DENSE (leaf pass only): the variant for trees whose fullest leaf holds at
// least kDenseSwitch particles or whose leaf capacity is kDenseCap or more,
// which hands full leaves to k_dense_p2p.  Both
// variants are launched; each returns at once unless the tree is its kind.
// XL (leaf pass only): the variant that also serves chain groups and
// streamed P2P, launched only when the near lists stop short of the deepest
// level or the P2P is streamed, so the other variants keep their registers.
// The plain sparse leaf variant (the reference's tree and far field) keeps
// 7 blocks per SM (72 registers), the order-1 leaf variants 4 (128).
template <int MODE, bool DEBUG, bool GRAD, bool DENSE, bool XL>
__global__ void __launch_bounds__(
    kTravThreads, (MODE == MODE_LEAF && !DEBUG && !XL) ? (GRAD ? 4 : (DENSE ? 1 : 7)) : 1)
    k_trav(TravArgs A) {
    using Smem = typename SmemOf<MODE>::T;
    __shared__ Smem smem[kTravWarps];
    const uint32_t lane = lane_id();
    const uint32_t lt_mask = lanemask_lt();
    Smem& sm = smem[threadIdx.x >> 5];
    const TreeView& tv = A.tv;
    Status* status = A.status;
    if (status->err & (PSG_ERR_NODES | PSG_ERR_SORT_SPIN)) return;
    // a run whose near lists ran out is void (the host grows them and runs
    // again): the internal levels below the one that failed did not run, so
    // their lists must not be read
    if (MODE == MODE_LEAF && (status->err & PSG_ERR_NS_OVERFLOW)) return;
    // the variant for this tree (batched systems: each group takes its
    // system's variant, so a system sums exactly as it does alone)
    if (MODE == MODE_LEAF && !tv.part_sys &&
        ((status->max_leaf >= kDenseSwitch || A.leaf_cap >= kDenseCap) != DENSE))
        return;
    // a shallower level's near lists did not fit: this level's are void
    if (MODE == MODE_INTERNAL && (status->ns_fail & ((1u << A.level) - 1u))) return;
    const float theta2 = __fmul_rn(A.theta, A.theta);

    // group index space: MODE_INTERNAL = the nodes at depth k-1; MODE_LEAF =
    // the nodes at depths 0..9, level after level
    uint32_t cum[kMaxDepth + 1];
    uint32_t total = 0;
    uint32_t* work;
    if (MODE == MODE_INTERNAL) {
        total = status->lvl_count[A.level - 1];
        work = &status->work[A.level];
    } else {
#pragma unroll
        for (int d = 0; d < kMaxDepth; ++d) {
            cum[d] = total;
            total += status->lvl_count[d];
        }
        cum[kMaxDepth] = total;
        // batched systems run both variants over all groups, each with its
        // own counter (work[1] is no internal level's); one system: work[0]
        work = &status->work[(tv.part_sys && DENSE) ? 1 : 0];
    }
    if (lane == 0) {
        if constexpr (MODE == MODE_INTERNAL) {
            sm.ns_next = 0;
            sm.ns_end = 0;
        } else {
            sm.chunk_next = 0;
            sm.chunk_end = 0;
        }
    }
    __syncwarp();
    // items taken per atomic: whole work queues are a few items per warp, so
    // the leaf pass takes them one by one (a batch would leave warps idle)
    const uint32_t batch = MODE == MODE_INTERNAL ? 4u : 1u;
    // the closure's order-1 accumulators take a group's children 4 at a time:
    // a work item is (group, half)
    constexpr uint32_t SL = GRAD ? 4u : 8u;
    constexpr uint32_t NH = 8u / SL;
    const uint32_t items = total * NH;

    for (;;) {
        uint32_t g0 = 0;
        if (lane == 0) g0 = atomicAdd(work, batch);
        g0 = __shfl_sync(0xFFFFFFFFu, g0, 0);
        if (g0 >= items) break;
#pragma unroll 1
        for (uint32_t gi = g0; gi < g0 + batch && gi < items; ++gi) {
            const uint32_t g = gi / NH, base = (gi % NH) * SL;
            uint32_t pid, dp;
            if (MODE == MODE_INTERNAL) {
                dp = A.level - 1;
                pid = tv.lvl_base[dp] + g;
            } else {
                dp = 0;
                uint32_t off = 0;
#pragma unroll
                for (int d = 1; d < kMaxDepth; ++d) {
                    if (g >= cum[d]) {
                        dp = d;
                        off = cum[d];
                    }
                }
                pid = tv.lvl_base[dp] + (g - off);
            }
            const long long t_group = DEBUG ? clock64() : 0;
            const uint32_t plink = tv.link[pid];
            const uint32_t nc = plink >> 28;
            if (nc == 0) continue;
            const uint32_t fc = plink & kLinkMask;
            // batched systems: the group's own system, theta and root; its
            // shallow leaves belong to k_heavy_leaf
            uint32_t gsys = 0;
            float th2 = theta2;
            if (tv.part_sys) {
                gsys = tv.part_sys[tv.info[pid].x];
                th2 = tv.sys_theta2[gsys];
                if (MODE == MODE_LEAF &&
                    ((int)dp < tv.sys_heavy[gsys] ||
                     ((tv.sys_maxleaf[gsys] >= kDenseSwitch || tv.sys_cap[gsys] >= kDenseCap) !=
                      DENSE)))
                    continue;
            }
            uint32_t cl = 0;
            if (lane < nc) {
                sm.cgeo[lane] = tv.geo[fc + lane];
                cl = tv.link[fc + lane];
            }
            cgp_put(sm.cgp, sm.cgeo, nc);
            const uint32_t leaf_mask =
                __ballot_sync(0xFFFFFFFFu, lane < nc && (cl >> 28) == 0) & 0xFFu;
            const uint32_t tgt_mask =
                (MODE == MODE_INTERNAL ? (((1u << nc) - 1u) & ~leaf_mask) : leaf_mask) &
                (((1u << SL) - 1u) << base);
            if (tgt_mask == 0) continue;
            if constexpr (MODE == MODE_LEAF) {
                if ((tgt_mask >> lane) & 1u) {
                    const uint4 ci = tv.info[fc + lane];
                    sm.cpart[lane] = make_uint2(ci.x, ci.y);
                }
            }
            if (lane < 8) {
                if (DEBUG) sm.dbg_m2l[lane] = 0;
                if constexpr (MODE == MODE_INTERNAL) {
                    sm.ns_cnt[lane] = 0;
                } else {
                    if (DEBUG) sm.dbg_p2p[lane] = 0;
                }
            }
            // chain group (leaf pass, parent deeper than the near lists
            // reach, K = ns_levels): start from the near list of p's ancestor
            // a at depth K and test its candidates down p's ancestor chain
            // a_{K+1} .. a_dp = p, as the reference's pair recursion does
            // (polesitter.h:1097-1145); what p is not separated from is
            // opened for the leaf children.  No near list below depth K is
            // stored, so nothing grows with theta.
            uint32_t nchain = 0, bnode = pid;
            if constexpr (MODE == MODE_LEAF) {
                if (XL && (int)dp > A.ns_levels) {
                    nchain = dp - (uint32_t)A.ns_levels;
                    uint32_t a = pid;
                    if (lane == 0) {
                        for (uint32_t c = nchain; c > 0; --c) {
                            sm.chain_geo[c - 1] = tv.geo[a];
                            a = tv.parent[a];
                        }
                    }
                    bnode = __shfl_sync(0xFFFFFFFFu, a, 0);
                    __syncwarp();
                    if (GRAD) {
                        // order 1 needs every ancestor's own gradient: chain
                        // groups serve the reference's order 0 only
                        if (lane == 0) set_err(status, PSG_ERR_CHAIN_ORDER);
                        continue;
                    }
                }
            }
            const float4 Lp = tv.lt[bnode];
            const bool root_only = dp <= 1;
            const uint32_t* nsl = nullptr;
            uint32_t nsn = 0;
            if (!root_only) {
                nsl = A.ns + tv.ns_off[bnode];
                nsn = tv.ns_cnt[bnode];
            }
            // MODE_INTERNAL: reserve |cand| near-list entries per target child
            uint32_t cand_total = 1;
            unsigned long long ns_base = 0;
            bool ns_ok = true;
            if constexpr (MODE == MODE_INTERNAL) {
                if (!root_only) {
                    uint32_t c = 0;
                    for (uint32_t e = lane; e < nsn; e += 32) {
                        const uint32_t nch = tv.link[nsl[e]] >> 28;
                        c += nch ? nch : 1u;
                    }
                    cand_total = warp_sum(c);
                }
                const unsigned long long need =
                    (unsigned long long)__popc(tgt_mask) * cand_total;
                __syncwarp();
                if (need && sm.ns_next + need > sm.ns_end) {
                    const unsigned long long take = need > kNsPool ? need : kNsPool;
                    unsigned long long b = 0;
                    if (lane == 0) b = atomicAdd(&status->ns_used[0], take);
                    b = __shfl_sync(0xFFFFFFFFu, b, 0);
                    __syncwarp();
                    if (lane == 0) {
                        sm.ns_next = b;
                        sm.ns_end = b + take;
                    }
                    __syncwarp();
                }
                ns_base = sm.ns_next;
                ns_ok = ns_base + need <= A.ns_cap;
                if (!ns_ok && lane == 0) {
                    set_err(status, PSG_ERR_NS_OVERFLOW);
                    atomicOr(&status->ns_fail, 1u << A.level);
                }
                __syncwarp();
                if (lane == 0) sm.ns_next = ns_base + need;
            }
            __syncwarp();

            // per pair of children (2k, 2k + 1): field and, for order 1, its
            // gradient, one child in each half of a float2
            float2 acc[SL / 2][3];
#pragma unroll
            for (int k = 0; k < (int)SL / 2; ++k)
                acc[k][0] = acc[k][1] = acc[k][2] = make_float2(0.f, 0.f);
            float2 gacc[GRAD ? SL / 2 : 1][6];
            if constexpr (GRAD) {
#pragma unroll
                for (int k = 0; k < (int)SL / 2; ++k)
#pragma unroll
                    for (int c = 0; c < 6; ++c) gacc[k][c] = make_float2(0.f, 0.f);
            }
            uint32_t ssize = 0, e0 = 0;
            uint32_t pfill = 0, phead = kNone;  // MODE_LEAF: staged / spilled P2P sources
            bool root_pending = root_only;
            float cacc0 = 0.f, cacc1 = 0.f, cacc2 = 0.f;  // chain groups: ancestors' M2L
            bool flushed = false;                         // STREAM: a flush has run
            unsigned long long sinter = 0;                // ... its pairs (debug)

            for (;;) {
                // ---- next batch of candidates into cand[0, tot) ----
                uint32_t tot;
                if (root_pending) {
                    if (lane == 0) {
                        sm.cand_node[0] = gsys;  // the (system's) root
                        sm.cand_mask[0] = (uint8_t)tgt_mask;
                        if constexpr (MODE == MODE_LEAF && XL) sm.cand_lvl[0] = 0;
                    }
                    tot = 1;
                    root_pending = false;
                } else if (e0 < nsn &&
                           (MODE == MODE_INTERNAL ||
                            ssize <= (uint32_t)(kStackCap - kStackSlack - kCandBuf))) {
                    const uint32_t e = e0 + lane;
                    uint32_t s0 = 0, c = 0, link = 0;
                    if (e < nsn) {
                        s0 = nsl[e];
                        link = tv.link[s0];
                        const uint32_t nch = link >> 28;
                        c = nch ? nch : 1u;
                    }
                    const uint32_t inc = warp_incl_scan(c);
                    tot = __shfl_sync(0xFFFFFFFFu, inc, 31);
                    const uint32_t ex = inc - c;
                    const bool lf = (link >> 28) == 0;
                    // a chain group's candidates are first tested against its
                    // ancestor a_{K+1} alone (level 1, no children)
                    const uint8_t cmk = (uint8_t)((XL && nchain) ? 0u : tgt_mask);
                    for (uint32_t i = 0; i < c; ++i) {
                        sm.cand_node[ex + i] = lf ? s0 : (link & kLinkMask) + i;
                        sm.cand_mask[ex + i] = cmk;
                        if constexpr (MODE == MODE_LEAF && XL)
                            sm.cand_lvl[ex + i] = nchain ? 1 : 0;
                    }
                    e0 += 32;
                } else if (MODE == MODE_LEAF && ssize > 0) {
                    // pop entries (bounded so the stack cannot overflow) and
                    // open them: an internal node's candidates are its
                    // children, a leaf's (pushed by a chain test) itself
                    const int room = ((int)kStackCap - kStackSlack - (int)ssize) / 7;
                    const uint32_t kp = (uint32_t)min(32, min((int)ssize, max(1, room)));
                    uint32_t node = 0, mask = 0, lvl = 0;
                    if constexpr (MODE == MODE_LEAF) {
                        if (lane < kp) {
                            node = sm.stk_node[ssize - kp + lane];
                            mask = sm.stk_mask[ssize - kp + lane];
                            if constexpr (XL) lvl = sm.stk_lvl[ssize - kp + lane];
                        }
                    }
                    __syncwarp();
                    ssize -= kp;
                    const uint32_t link = lane < kp ? tv.link[node] : 0u;
                    const uint32_t nch = link >> 28;
                    const uint32_t c = lane < kp ? (XL && nch == 0 ? 1u : nch) : 0u;
                    const uint32_t inc = warp_incl_scan(c);
                    tot = __shfl_sync(0xFFFFFFFFu, inc, 31);
                    const uint32_t ex = inc - c;
                    for (uint32_t i = 0; i < c; ++i) {
                        sm.cand_node[ex + i] = nch ? (link & kLinkMask) + i : node;
                        sm.cand_mask[ex + i] = (uint8_t)mask;
                        if constexpr (MODE == MODE_LEAF && XL) sm.cand_lvl[ex + i] = (uint8_t)lvl;
                    }
                } else {
                    break;
                }
                __syncwarp();

                // ---- test the candidates, one per lane; the next chunk's node
                // records are loaded while the current one is processed ----
                uint32_t n_s = 0, n_mask = 0, n_link = 0, n_lvl = 0;
                float4 n_g = make_float4(0.f, 0.f, 0.f, 0.f), n_mp = n_g;
                if (lane < tot) {
                    n_s = sm.cand_node[lane];
                    n_mask = sm.cand_mask[lane];
                    if constexpr (MODE == MODE_LEAF && XL) n_lvl = sm.cand_lvl[lane];
                    n_g = tv.geo[n_s];
                    n_mp = tv.mp[n_s];
                    n_link = tv.link[n_s];
                }
#pragma unroll 1
                for (uint32_t j0 = 0; j0 < tot; j0 += 32) {
                    const uint32_t s = n_s, smask = n_mask, slink = n_link, slvl = n_lvl;
                    const float4 sg = n_g, smp = n_mp;
                    {
                        const uint32_t jn = j0 + 32 + lane;
                        n_mask = 0;
                        n_lvl = 0;
                        if (jn < tot) {
                            n_s = sm.cand_node[jn];
                            n_mask = sm.cand_mask[jn];
                            if constexpr (MODE == MODE_LEAF && XL) n_lvl = sm.cand_lvl[jn];
                            n_g = tv.geo[n_s];
                            n_mp = tv.mp[n_s];
                            n_link = tv.link[n_s];
                        }
                    }
                    const uint32_t chunk_mask = __reduce_or_sync(0xFFFFFFFFu, smask);
                    uint32_t near_bits = 0;
                    // children two at a time: the MAC per child (mac_separated,
                    // scalar, so its decisions are the reference's), then the
                    // M2L of m2l_field(_grad) for both children in paired FP32
                    // instructions, each half rounding as the scalar form does
#pragma unroll
                    for (uint32_t k = 0; k < SL / 2; ++k) {
                        const uint32_t q = base + 2 * k;  // children q and q + 1
                        if (!((chunk_mask >> q) & 3u)) continue;
                        const float4 ga = sm.cgp[q >> 1][0], gb = sm.cgp[q >> 1][1];
                        float dx0, dy0, dz0, e0, dx1, dy1, dz1, e1;
                        const bool m0 = mac_separated(ga.x, ga.z, gb.x, gb.z, sg.x, sg.y, sg.z,
                                                      sg.w, th2, dx0, dy0, dz0, e0);
                        const bool m1 = mac_separated(ga.y, ga.w, gb.y, gb.w, sg.x, sg.y, sg.z,
                                                      sg.w, th2, dx1, dy1, dz1, e1);
                        const float2 dx = make_float2(dx0, dx1), dy = make_float2(dy0, dy1),
                                     dz = make_float2(dz0, dz1), d2 = make_float2(e0, e1);
                        const bool a0 = (smask >> q) & 1u, a1 = (smask >> (q + 1)) & 1u;
                        const bool s0 = m0 && a0, s1 = m1 && a1;
                        // branch-free: every lane evaluates, only separated
                        // pairs add (x * 1 + acc = x + acc, x * 0 + acc = acc)
                        const float2 on = make_float2(s0 ? 1.f : 0.f, s1 ? 1.f : 0.f);
                        const float2 soft = __fadd2_rn(d2, make_float2(0.1f, 0.1f));
                        const float2 inv = make_float2(rsqrtf(soft.x), rsqrtf(soft.y));
                        const float2 inv2 = __fmul2_rn(inv, inv);
                        const float2 ir3 = __fmul2_rn(inv2, inv);
                        const float2 ir5 = __fmul2_rn(ir3, inv2);
                        const float2 mx = make_float2(smp.x, smp.x),
                                     my = make_float2(smp.y, smp.y),
                                     mz = make_float2(smp.z, smp.z),
                                     mw = make_float2(smp.w, smp.w);
                        const float2 mdr =
                            __ffma2_rn(my, dx, __ffma2_rn(mz, dy, __fmul2_rn(mw, dz)));
                        const float2 a = __ffma2_rn(
                            mx, ir3, __fmul2_rn(__fmul2_rn(make_float2(-3.f, -3.f), mdr), ir5));
                        const float2 fx = __ffma2_rn(dx, a, __fmul2_rn(my, ir3));
                        const float2 fy = __ffma2_rn(dy, a, __fmul2_rn(mz, ir3));
                        const float2 fz = __ffma2_rn(dz, a, __fmul2_rn(mw, ir3));
                        acc[k][0] = __ffma2_rn(fx, on, acc[k][0]);
                        acc[k][1] = __ffma2_rn(fy, on, acc[k][1]);
                        acc[k][2] = __ffma2_rn(fz, on, acc[k][2]);
                        if constexpr (GRAD) {
                            // g3 d d^T - gi I, g3 = 3 m0 / r^5, gi = m0 / r^3
                            const float2 g3 = __fmul2_rn(
                                __fmul2_rn(__fmul2_rn(make_float2(3.f, 3.f), mx), ir5), on);
                            const float2 gi = __fmul2_rn(__fmul2_rn(mx, ir3), on);
                            const float2 ngi = make_float2(-gi.x, -gi.y);
                            const float2 gx = __fmul2_rn(g3, dx), gy = __fmul2_rn(g3, dy);
                            gacc[k][0] = __fadd2_rn(gacc[k][0], __ffma2_rn(gx, dx, ngi));
                            gacc[k][1] = __fadd2_rn(gacc[k][1], __ffma2_rn(gy, dy, ngi));
                            gacc[k][2] = __fadd2_rn(gacc[k][2],
                                                    __ffma2_rn(__fmul2_rn(g3, dz), dz, ngi));
                            gacc[k][3] = __ffma2_rn(gx, dy, gacc[k][3]);
                            gacc[k][4] = __ffma2_rn(gx, dz, gacc[k][4]);
                            gacc[k][5] = __ffma2_rn(gy, dz, gacc[k][5]);
                        }
                        if (a0 && !s0) near_bits |= 1u << q;
                        if (a1 && !s1) near_bits |= 2u << q;
                        if (DEBUG) {
                            const uint32_t b0 = __ballot_sync(0xFFFFFFFFu, s0);
                            const uint32_t b1 = __ballot_sync(0xFFFFFFFFu, s1);
                            if (lane == 0) {
                                sm.dbg_m2l[q] += __popc(b0);
                                sm.dbg_m2l[q + 1] += __popc(b1);
                            }
                        }
                    }
                    if constexpr (MODE == MODE_INTERNAL) {
                        // near candidates of internal children: their near lists
                        const uint32_t near_any = __reduce_or_sync(0xFFFFFFFFu, near_bits);
#pragma unroll 1
                        for (uint32_t m = near_any; m; m &= m - 1) {
                            const uint32_t q = __ffs(m) - 1;
                            const bool nr = (near_bits >> q) & 1u;
                            const uint32_t nm = __ballot_sync(0xFFFFFFFFu, nr);
                            const uint32_t base = sm.ns_cnt[q];
                            if (ns_ok && nr) {
                                const uint32_t sub = __popc(tgt_mask & ((1u << q) - 1u));
                                A.ns[ns_base + (unsigned long long)sub * cand_total + base +
                                     __popc(nm & lt_mask)] = s;
                            }
                            __syncwarp();
                            if (lane == 0) sm.ns_cnt[q] = base + __popc(nm);
                            __syncwarp();
                        }
                    } else {
                        const bool sleaf = (slink >> 28) == 0;
                        // chain candidates: the MAC against their ancestor
                        // target; separated -> M2L into the chain's field,
                        // else opened for the next ancestor (past p: for the
                        // leaf children, with the whole target mask)
                        bool cpush = false;
                        uint32_t cmask = 0, clvl = 0;
                        if (XL && nchain && __any_sync(0xFFFFFFFFu, slvl != 0)) {
                            if (slvl) {
                                const float4 cg = sm.chain_geo[slvl - 1];
                                float dx, dy, dz, d2;
                                if (mac_separated(cg.x, cg.y, cg.z, cg.w, sg.x, sg.y, sg.z, sg.w,
                                                  th2, dx, dy, dz, d2)) {
                                    float fx, fy, fz;
                                    m2l_field(dx, dy, dz, d2, smp, fx, fy, fz);
                                    cacc0 += fx;
                                    cacc1 += fy;
                                    cacc2 += fz;
                                } else {
                                    cpush = true;
                                    cmask = slvl == nchain ? tgt_mask : 0u;
                                    clvl = slvl == nchain ? 0u : slvl + 1;
                                }
                            }
                        }
                        // near leaf candidate: a P2P source of these children
                        const uint32_t pbits = sleaf ? near_bits : 0u;
                        const uint32_t pb = __ballot_sync(0xFFFFFFFFu, pbits != 0);
                        if (pb) {
                            if (pfill + __popc(pb) > (uint32_t)kP2PCap) {
                                if (XL && A.stream) {
                                    stream_p2p<DEBUG, GRAD>(
                                        sm,
                                        LeafOut{A.xyzm, tv.info, A.p2p, A.fx, A.fy, A.fz,
                                                A.leaf_of, tv.dbg_p2p, A.dense_rec, A.dense_cap,
                                                A.kahan},
                                        tgt_mask, fc, pfill, flushed, false, sinter);
                                    flushed = true;
                                } else {
                                    phead = spill_p2p(sm, pfill, phead, A.p2p, status);
                                }
                                pfill = 0;
                            }
                            if (pbits) {
                                const uint32_t pos = pfill + __popc(pb & lt_mask);
                                sm.p2p_node[pos] = s;
                                sm.p2p_mask[pos] = (uint8_t)pbits;
                            }
                            pfill += __popc(pb);
                            if (DEBUG) {
                                const uint32_t pany = __reduce_or_sync(0xFFFFFFFFu, pbits);
                                for (uint32_t m = pany; m; m &= m - 1) {
                                    const uint32_t q = __ffs(m) - 1;
                                    const uint32_t c =
                                        __popc(__ballot_sync(0xFFFFFFFFu, (pbits >> q) & 1u));
                                    if (lane == 0) sm.dbg_p2p[q] += c;
                                }
                            }
                        }
                        // near internal candidate: open it later for these children
                        const uint32_t qbits = sleaf ? 0u : near_bits;
                        const bool push = qbits != 0 || cpush;
                        const uint32_t qb = __ballot_sync(0xFFFFFFFFu, push);
                        if (qb) {
                            const uint32_t pos = ssize + __popc(qb & lt_mask);
                            if (push && pos < (uint32_t)kStackCap) {
                                sm.stk_node[pos] = s;
                                sm.stk_mask[pos] = (uint8_t)(cpush ? cmask : qbits);
                                if constexpr (XL) sm.stk_lvl[pos] = (uint8_t)(cpush ? clvl : 0u);
                            }
                            ssize += __popc(qb);
                            if (ssize > (uint32_t)kStackCap) {
                                if (lane == 0) set_err(status, PSG_ERR_STACK);
                                ssize = kStackCap;
                            }
                        }
                    }
                    __syncwarp();
                }
                if (MODE == MODE_LEAF && DEBUG && lane == 0) atomicMax(&status->max_stack, ssize);
            }

            // ---- L2L: L(u) = M2L(u) + L(parent)  (polesitter.h:1248-1250) ----
            // closure order 1 shifts the parent's field to the child's centre:
            // L(u) = M2L(u) + L(p) + G(p) (c_u - c_p), G(u) = M2L_G(u) + G(p).
            // A chain group's parent field is L(a) + the chain's M2L.
            float4 Lb = Lp;
            if (XL && nchain) {
                Lb.y = __fadd_rn(Lb.y, warp_sum(cacc0));
                Lb.z = __fadd_rn(Lb.z, warp_sum(cacc1));
                Lb.w = __fadd_rn(Lb.w, warp_sum(cacc2));
            }
            float4 Gp0 = make_float4(0.f, 0.f, 0.f, 0.f), cp = Gp0;
            float2 Gp1 = make_float2(0.f, 0.f);
            if constexpr (GRAD) {
                cp = tv.geo[pid];
                if (dp >= 2) {
                    Gp0 = tv.lg0[pid];
                    Gp1 = tv.lg1[pid];
                }
            }
#pragma unroll
            for (uint32_t k = 0; k < SL; ++k) {
                const uint32_t q = base + k;
                if (!((tgt_mask >> q) & 1u)) continue;
                const float2* ak = acc[k >> 1];
                const float ax = warp_sum((k & 1) ? ak[0].y : ak[0].x);
                const float ay = warp_sum((k & 1) ? ak[1].y : ak[1].x);
                const float az = warp_sum((k & 1) ? ak[2].y : ak[2].x);
                float4 L = make_float4(0.f, __fadd_rn(ax, Lb.y), __fadd_rn(ay, Lb.z),
                                       __fadd_rn(az, Lb.w));
                float4 G0 = Gp0;
                float2 G1 = Gp1;
                if constexpr (GRAD) {
                    const float4 cu = sm.cgeo[q];
                    const float3 sh = grad_apply(Gp0, Gp1, cu.x - cp.x, cu.y - cp.y, cu.z - cp.z);
                    L.y += sh.x;
                    L.z += sh.y;
                    L.w += sh.z;
                    const float2* gk = gacc[k >> 1];
                    G0.x += warp_sum((k & 1) ? gk[0].y : gk[0].x);
                    G0.y += warp_sum((k & 1) ? gk[1].y : gk[1].x);
                    G0.z += warp_sum((k & 1) ? gk[2].y : gk[2].x);
                    G0.w += warp_sum((k & 1) ? gk[3].y : gk[3].x);
                    G1.x += warp_sum((k & 1) ? gk[4].y : gk[4].x);
                    G1.y += warp_sum((k & 1) ? gk[5].y : gk[5].x);
                }
                if (lane == 0) {
                    const uint32_t u = fc + q;
                    tv.lt[u] = L;
                    if constexpr (GRAD) {
                        tv.lg0[u] = G0;
                        tv.lg1[u] = G1;
                    }
                    if constexpr (MODE == MODE_LEAF) {
                        sm.sL[q] = L;
                        if constexpr (GRAD) {
                            sm.sG0[q] = G0;
                            sm.sG1[q] = G1;
                        }
                    } else {
                        const uint32_t sub = __popc(tgt_mask & ((1u << q) - 1u));
                        tv.ns_off[u] = (uint32_t)(ns_base + (unsigned long long)sub * cand_total);
                        tv.ns_cnt[u] = ns_ok ? sm.ns_cnt[q] : 0u;
                    }
                    if (DEBUG) {
                        tv.dbg_m2l[u] = sm.dbg_m2l[q];
                        atomicAdd(&status->stat[PSG_STAT_M2L], (unsigned long long)sm.dbg_m2l[q]);
                    }
                }
            }
            __syncwarp();

            if constexpr (MODE == MODE_LEAF) {
                leaf_epilogue<DEBUG, GRAD, DENSE>(
                    sm,
                    LeafOut{A.xyzm, tv.info, A.p2p, A.fx, A.fy, A.fz, A.leaf_of, tv.dbg_p2p,
                            A.dense_rec, A.dense_cap, A.kahan},
                    tgt_mask, fc, pfill, phead, XL && A.stream != 0, flushed, sinter, status);
                if (DEBUG && lane == 0) {
                    const unsigned long long cyc = (unsigned long long)(clock64() - t_group);
                    atomicMax(&status->stat[PSG_STAT_SLOWEST_GROUP],
                              (min(cyc, (1ull << 36) - 1) << 28) | pid);
                }
            }
        }
    }
}

// L2P + P2P of the full leaves recorded by the leaf pass.  A warp takes one
// record (a run of leaves, up to 32 of their particles, the group's source
// chain) at a time from a shared counter.  The chain's entries (source
// leaves) are split by the leaves of the record they serve:
//  * an entry that serves every leaf of the record is summed by all lanes:
//    T lanes own the record's target particles (T the smallest power of two
//    >= their count) and the 32 / T slices of lanes split the entry's
//    particles;
//  * an entry that serves only some of its leaves is summed per leaf q, in
//    another walk of the chain, with the lanes dealt over q's targets alone
//    (T_q lanes, 32 / T_q slices),
// so no lane computes a pair its target does not want.  A chunk's taken
// entries go through the warp's shared tile (sum_tiles); with 8 or more
// slices (4 or fewer targets) the slices instead walk whole source leaves
// from global memory (walk_leaf), as the tile's search would cost more than
// its reuse saves.  The per-leaf sums reach the target's lane through
// shared memory (a target belongs to one leaf, so its slot is written once).
// Sums are taken in chain order, so the result does not depend on
// scheduling.

// A tile of 32 source particles, pair-packed: pair m holds particles 2m and
// 2m + 1 as a = {x, x', y, y'} and b = {z, z', w, w'}, so one 128-bit
// shared load gives two sources' coordinates as the float2 operands of
// sm_100's paired FP32 instructions (__fadd2_rn, __ffma2_rn, __fmul2_rn):
// one issued instruction does a step of two pairs.
struct DenseTile {
    float4 a[16];
    float4 b[16];
};

__device__ __forceinline__ void tile_put(DenseTile& tile, uint32_t lane, float4 p) {
    float* a = reinterpret_cast<float*>(&tile.a[lane >> 1]);
    float* b = reinterpret_cast<float*>(&tile.b[lane >> 1]);
    const uint32_t h = lane & 1u;
    a[h] = p.x;
    a[2 + h] = p.y;
    b[h] = p.z;
    b[2 + h] = p.w;
}

// one target against the tile's source pairs m = m0, m0 + S, ... (sources
// 2m and 2m + 1, fewer than nt real ones; the slot past an odd nt holds a
// zero mass, which adds exactly zero).  Plain sums keep the two sources of
// a pair in the two halves of float2 accumulators (two FMA chains in one
// instruction); Kahan sums go source by source.
template <bool KAHAN>
__device__ __forceinline__ void dense_tile(const DenseTile& tile, uint32_t m0, uint32_t S,
                                           uint32_t nt, float4 t, float2& sx, float2& sy,
                                           float2& sz, float& ax, float& ay, float& az,
                                           float& cx, float& cy, float& cz) {
    if constexpr (KAHAN) {
        for (uint32_t m = m0; 2 * m < nt; m += S) {
            const float4 a = tile.a[m], b = tile.b[m];
            for (uint32_t h = 0; h < 2 && 2 * m + h < nt; ++h) {
                const float px = h ? a.y : a.x, py = h ? a.w : a.z, pz = h ? b.y : b.x,
                            pw = h ? b.w : b.z;
                const float dx = px - t.x, dy = py - t.y, dz = pz - t.z;
                const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz)) + 0.1f;
                const float inv = rsqrtf(r2);
                const float f = pw * (inv * inv * inv);
                const float yx = __fsub_rn(__fmul_rn(dx, f), cx);
                const float yy = __fsub_rn(__fmul_rn(dy, f), cy);
                const float yz = __fsub_rn(__fmul_rn(dz, f), cz);
                const float tx = __fadd_rn(ax, yx);
                const float ty = __fadd_rn(ay, yy);
                const float tz = __fadd_rn(az, yz);
                cx = __fsub_rn(__fsub_rn(tx, ax), yx);
                cy = __fsub_rn(__fsub_rn(ty, ay), yy);
                cz = __fsub_rn(__fsub_rn(tz, az), yz);
                ax = tx;
                ay = ty;
                az = tz;
            }
        }
    } else {
        const float2 ntx = make_float2(-t.x, -t.x), nty = make_float2(-t.y, -t.y),
                     ntz = make_float2(-t.z, -t.z), eps = make_float2(0.1f, 0.1f);
        const uint32_t np = (nt + 1u) >> 1;
#pragma unroll 2
        for (uint32_t m = m0; m < np; m += S) {
            const float4 a = tile.a[m], b = tile.b[m];
            const float2 dx = __fadd2_rn(make_float2(a.x, a.y), ntx);
            const float2 dy = __fadd2_rn(make_float2(a.z, a.w), nty);
            const float2 dz = __fadd2_rn(make_float2(b.x, b.y), ntz);
            float2 r = __ffma2_rn(dz, dz, eps);
            r = __ffma2_rn(dy, dy, r);
            r = __ffma2_rn(dx, dx, r);
            const float2 i = make_float2(rsqrtf(r.x), rsqrtf(r.y));
            const float2 f = __fmul2_rn(make_float2(b.z, b.w), __fmul2_rn(__fmul2_rn(i, i), i));
            sx = __ffma2_rn(dx, f, sx);
            sy = __ffma2_rn(dy, f, sy);
            sz = __ffma2_rn(dz, f, sz);
        }
    }
}

// The particles of the chunk entries the lanes hold (entry start es, count
// en; en = 0 for an entry not taken) against target t: laid end to end by a
// warp prefix sum, they pass through the warp's shared tile 32 at a time --
// lane j finds the entry of flat particle b + j by a binary search over the
// prefix sums and stages it (coalesced within a leaf) -- and every lane runs
// its target against the tile's source pairs m = slice, slice + S, ...
// Returns the particles summed (the same on every lane).
template <bool KAHAN>
__device__ __forceinline__ uint32_t sum_tiles(DenseTile& tile, const float4* __restrict__ xyzm,
                                              uint32_t es, uint32_t en, uint32_t slice,
                                              uint32_t S, float4 t, float& ax, float& ay,
                                              float& az, float& cx, float& cy, float& cz) {
    const uint32_t lane = lane_id();
    const uint32_t incl = warp_incl_scan(en);
    const uint32_t ptot = __shfl_sync(0xFFFFFFFFu, incl, 31);
    const uint32_t excl = incl - en;
    // lane j's particle of the tile starting at flat index b (warp-collective)
    auto fetch = [&](uint32_t b) -> float4 {
        const uint32_t f = b + lane;
        uint32_t e = 0;
#pragma unroll
        for (uint32_t step = 16; step > 0; step >>= 1) {
            const uint32_t v = __shfl_sync(0xFFFFFFFFu, incl, e + step - 1);
            if (v <= f) e += step;
        }
        const uint32_t e_start = __shfl_sync(0xFFFFFFFFu, es, e);
        const uint32_t e_excl = __shfl_sync(0xFFFFFFFFu, excl, e);
        return f < ptot ? xyzm[e_start + (f - e_excl)] : make_float4(0.f, 0.f, 0.f, 0.f);
    };
    float2 sx = make_float2(0.f, 0.f), sy = sx, sz = sx;
    float4 pcur = ptot ? fetch(0u) : make_float4(0.f, 0.f, 0.f, 0.f);
    for (uint32_t b = 0; b < ptot; b += 32) {
        __syncwarp();
        tile_put(tile, lane, pcur);
        __syncwarp();
        // the next tile's particle is in flight while this tile is summed
        if (b + 32 < ptot) pcur = fetch(b + 32);
        const uint32_t nt = min(32u, ptot - b);
        dense_tile<KAHAN>(tile, slice, S, nt, t, sx, sy, sz, ax, ay, az, cx, cy, cz);
    }
    __syncwarp();
    if constexpr (!KAHAN) {
        ax += sx.x + sx.y;
        ay += sy.x + sy.y;
        az += sz.x + sz.y;
    }
    return ptot;
}

// target t against the particles first + slice, first + slice + S, ... <
// first + cnt (polesitter.h:1424-1444, rsqrt), optionally Kahan-compensated
template <bool KAHAN>
__device__ __forceinline__ void walk_leaf(const float4* __restrict__ xyzm, uint32_t first,
                                          uint32_t cnt, uint32_t slice, uint32_t S, float4 t,
                                          float& ax, float& ay, float& az, float& cx,
                                          float& cy, float& cz) {
    if constexpr (KAHAN) {
        for (uint32_t j = slice; j < cnt; j += S) {
            const float4 p = xyzm[first + j];
            const float dx = p.x - t.x, dy = p.y - t.y, dz = p.z - t.z;
            const float inv = rsqrtf(fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, 0.1f))));
            const float f = p.w * (inv * inv * inv);
            const float yx = __fsub_rn(__fmul_rn(dx, f), cx);
            const float yy = __fsub_rn(__fmul_rn(dy, f), cy);
            const float yz = __fsub_rn(__fmul_rn(dz, f), cz);
            const float tx = __fadd_rn(ax, yx);
            const float ty = __fadd_rn(ay, yy);
            const float tz = __fadd_rn(az, yz);
            cx = __fsub_rn(__fsub_rn(tx, ax), yx);
            cy = __fsub_rn(__fsub_rn(ty, ay), yy);
            cz = __fsub_rn(__fsub_rn(tz, az), yz);
            ax = tx;
            ay = ty;
            az = tz;
        }
    } else {
        float ex = 0.f, ey = 0.f, ez = 0.f;
        uint32_t j = slice;
        for (; j + S < cnt; j += 2 * S) {
            const float4 p0 = xyzm[first + j], p1 = xyzm[first + j + S];
            const float dx0 = p0.x - t.x, dy0 = p0.y - t.y, dz0 = p0.z - t.z;
            const float dx1 = p1.x - t.x, dy1 = p1.y - t.y, dz1 = p1.z - t.z;
            const float i0 = rsqrtf(fmaf(dx0, dx0, fmaf(dy0, dy0, fmaf(dz0, dz0, 0.1f))));
            const float i1 = rsqrtf(fmaf(dx1, dx1, fmaf(dy1, dy1, fmaf(dz1, dz1, 0.1f))));
            const float f0 = p0.w * (i0 * i0 * i0), f1 = p1.w * (i1 * i1 * i1);
            ax = fmaf(dx0, f0, ax);
            ay = fmaf(dy0, f0, ay);
            az = fmaf(dz0, f0, az);
            ex = fmaf(dx1, f1, ex);
            ey = fmaf(dy1, f1, ey);
            ez = fmaf(dz1, f1, ez);
        }
        if (j < cnt) {
            const float4 p = xyzm[first + j];
            const float dx = p.x - t.x, dy = p.y - t.y, dz = p.z - t.z;
            const float inv = rsqrtf(fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, 0.1f))));
            const float f = p.w * (inv * inv * inv);
            ax = fmaf(dx, f, ax);
            ay = fmaf(dy, f, ay);
            az = fmaf(dz, f, az);
        }
        ax += ex;
        ay += ey;
        az += ez;
    }
}

// a spilled chunk as one lane sees it: the chunk's entry count and link,
// and the lane's entry (its source leaf and child mask; slots past the count
// hold stale values and are not used)
struct ChunkHead {
    uint32_t cnt, next, src, mask;
};

__device__ __forceinline__ ChunkHead load_chunk(const P2PStore& st, uint32_t c, uint32_t lane) {
    ChunkHead h{0u, kNone, 0u, 0u};
    if (c != kNone) {
        h.cnt = st.cnt[c];
        h.next = st.next[c];
        h.src = st.src[(size_t)c * kP2PChunk + lane];
        h.mask = st.mask[(size_t)c * kP2PChunk + lane];
    }
    return h;
}

template <bool DEBUG, bool GRAD, bool KAHAN>
__global__ void __launch_bounds__(kTravThreads, kDenseBlocksPerSm) k_dense_p2p(TravArgs A) {
    __shared__ float4 s_part[kTravWarps][32];  // per-leaf sums of the record's targets
    __shared__ DenseTile tiles[kTravWarps];
    __shared__ uint2 s_ent[kTravWarps][32];  // pass 2: a leaf's entries, 32 at a time
    float4* part = s_part[threadIdx.x >> 5];
    DenseTile& tile = tiles[threadIdx.x >> 5];
    uint2* ent = s_ent[threadIdx.x >> 5];
    // this warp's list of partial entries (source start, count | mask << 16)
    const uint32_t wslot = blockIdx.x * kTravWarps + (threadIdx.x >> 5);
    if (wslot >= A.dense_part_warps) return;  // (no list: the other warps take the records)
    uint2* const plist = A.dense_part + (size_t)wslot * kDensePartCap;
    Status* status = A.status;
    if (status->err & (PSG_ERR_NODES | PSG_ERR_SORT_SPIN | PSG_ERR_DENSE_OVERFLOW)) return;
    const TreeView& tv = A.tv;
    const float4* __restrict__ xyzm = A.xyzm;
    const uint32_t lane = lane_id();
    const uint32_t total = min(status->dense_count, A.dense_cap);
    if (total == 0) return;
    unsigned long long inter = 0;
    for (;;) {
        uint32_t r = 0;
        if (lane == 0) r = atomicAdd(&status->dense_work, 1u);
        r = __shfl_sync(0xFFFFFFFFu, r, 0);
        if (r >= total) break;
        const uint4 rec = A.dense_rec[r];
        const uint32_t fc = rec.x, run = rec.w >> 8, cnt_t = rec.w & 0xFFu, first = rec.z;
        uint32_t T = 1;
        while (T < cnt_t) T <<= 1;
        const uint32_t S = 32u / T;
        const uint32_t tl = lane & (T - 1u), slice = lane / T;
        const bool active = tl < cnt_t;
        const uint32_t i = first + (active ? tl : 0u);
        // this lane's leaf: the child of the run whose particles hold i
        uint32_t q = __ffs(run) - 1;
        for (uint32_t m = run; m; m &= m - 1) {
            const uint32_t qq = __ffs(m) - 1;
            if (tv.info[fc + qq].x <= i) q = qq;
        }
        const uint32_t u = fc + q;
        const float4 t = xyzm[i];
        part[lane] = make_float4(0.f, 0.f, 0.f, 0.f);
        __syncwarp();
        float bx = 0.f, by = 0.f, bz = 0.f, cx = 0.f, cy = 0.f, cz = 0.f;
        uint32_t used = 0;
        // The chain is walked once, in segments.  Pass 1 sums the entries
        // that serve every leaf of the record and keeps the others (partial
        // entries) in the warp's list, in chain order; when the list could
        // not take another chunk, or at the chain's end, pass 2 sums the
        // listed entries leaf by leaf and the list starts over.  While a
        // chunk is summed, the next chunk's source ranges and the header
        // after it are in flight.
        auto src_range = [&](const ChunkHead& hh) -> uint2 {
            if (lane < hh.cnt && (hh.mask & run) != 0u) {
                const uint4 si = tv.info[hh.src];
                return make_uint2(si.x, si.y);
            }
            return make_uint2(0u, 0u);
        };
        ChunkHead h = load_chunk(A.p2p, rec.y, lane);
        uint2 hr = src_range(h);
        ChunkHead hn = load_chunk(A.p2p, h.next, lane);
        uint32_t c = rec.y;
        for (;;) {
            uint32_t npart = 0, partial_q = 0;
            while (c != kNone && npart + 32u <= kDensePartCap) {
                const uint32_t em = lane < h.cnt ? (h.mask & run) : 0u;
                const uint32_t es = hr.x, en = hr.y;
                c = h.next;
                h = hn;
                hr = src_range(h);
                hn = load_chunk(A.p2p, h.next, lane);
                const bool partial = em != 0u && em != run;
                partial_q |= __reduce_or_sync(0xFFFFFFFFu, partial ? em : 0u);
                const uint32_t pb = __ballot_sync(0xFFFFFFFFu, partial);
                if (partial)
                    plist[npart + __popc(pb & ((1u << lane) - 1u))] =
                        make_uint2(es, en | (em << 16));
                npart += __popc(pb);
                if (S >= 8u) {
                    for (uint32_t full = __ballot_sync(0xFFFFFFFFu, em == run); full;
                         full &= full - 1) {
                        const uint32_t e = __ffs(full) - 1;
                        const uint32_t s0 = __shfl_sync(0xFFFFFFFFu, es, e);
                        const uint32_t n0 = __shfl_sync(0xFFFFFFFFu, en, e);
                        walk_leaf<KAHAN>(xyzm, s0, n0, slice, S, t, bx, by, bz, cx, cy, cz);
                        if (DEBUG) used += n0;
                    }
                } else {
                    const uint32_t got = sum_tiles<KAHAN>(tile, xyzm, es, em == run ? en : 0u,
                                                          slice, S, t, bx, by, bz, cx, cy, cz);
                    if (DEBUG) used += got;
                }
            }
            // pass 2: per leaf q of the record, its listed entries, gathered
            // 32 at a time in shared memory so that the tiles run full; the
            // lanes are dealt over q's targets alone (T_q lanes, 32 / T_q
            // slices)
            __syncwarp();
            for (uint32_t m = partial_q; m; m &= m - 1) {
                const uint32_t qq = __ffs(m) - 1;
                const uint4 ci = tv.info[fc + qq];
                const uint32_t lo = max(ci.x, first), hi = min(ci.x + ci.y, first + cnt_t);
                if (hi <= lo) continue;
                const uint32_t nq = hi - lo;
                uint32_t Tq = 1;
                while (Tq < nq) Tq <<= 1;
                const uint32_t Sq = 32u / Tq, tq = lane & (Tq - 1u), sq = lane / Tq;
                const bool actq = tq < nq;
                const uint32_t iq = lo + (actq ? tq : 0u);
                const float4 tp = xyzm[iq];
                float px = 0.f, py = 0.f, pz = 0.f, kx = 0.f, ky = 0.f, kz = 0.f;
                uint32_t usedq = 0, kept = 0;
                for (uint32_t b = 0;; b += 32) {
                    // take the next 32 listed entries' share for q; sum the
                    // gathered ones when 32 are in (or at the list's end)
                    const bool more = b < npart;
                    uint2 v = make_uint2(0u, 0u);
                    if (more && b + lane < npart) v = plist[b + lane];
                    const bool mine = (v.y >> (16 + qq)) & 1u;
                    const uint32_t mb = __ballot_sync(0xFFFFFFFFu, mine);
                    const uint32_t pos = kept + __popc(mb & ((1u << lane) - 1u));
                    const uint2 e2 = make_uint2(v.x, v.y & 0xFFFFu);
                    if (mine && pos < 32u) ent[pos] = e2;
                    kept += __popc(mb);
                    if (kept >= 32u || (!more && kept > 0u)) {
                        const uint32_t k = min(kept, 32u);
                        __syncwarp();
                        const uint2 g = lane < k ? ent[lane] : make_uint2(0u, 0u);
                        __syncwarp();
                        if (mine && pos >= 32u) ent[pos - 32u] = e2;
                        kept -= k;
                        if (Sq >= 8u) {
                            for (uint32_t pm = __ballot_sync(0xFFFFFFFFu, lane < k); pm;
                                 pm &= pm - 1) {
                                const uint32_t e = __ffs(pm) - 1;
                                const uint32_t s0 = __shfl_sync(0xFFFFFFFFu, g.x, e);
                                const uint32_t n0 = __shfl_sync(0xFFFFFFFFu, g.y, e);
                                walk_leaf<KAHAN>(xyzm, s0, n0, sq, Sq, tp, px, py, pz, kx, ky, kz);
                                if (DEBUG) usedq += n0;
                            }
                        } else {
                            const uint32_t got = sum_tiles<KAHAN>(tile, xyzm, g.x, g.y, sq, Sq, tp,
                                                                  px, py, pz, kx, ky, kz);
                            if (DEBUG) usedq += got;
                        }
                    }
                    if (!more) break;
                }
                px -= kx;
                py -= ky;
                pz -= kz;
                for (uint32_t o = Tq; o < 32u; o <<= 1) {
                    px += __shfl_xor_sync(0xFFFFFFFFu, px, o);
                    py += __shfl_xor_sync(0xFFFFFFFFu, py, o);
                    pz += __shfl_xor_sync(0xFFFFFFFFu, pz, o);
                }
                if (actq && sq == 0) {
                    float4& pp = part[iq - first];
                    pp.x += px;
                    pp.y += py;
                    pp.z += pz;
                }
                if (DEBUG) inter += (actq && sq == 0) ? usedq : 0u;
                __syncwarp();
            }
            if (c == kNone) break;
        }
        __syncwarp();
        if (DEBUG) inter += (active && slice == 0) ? used : 0u;
        // sum the slices' partial sums (fixed order)
        bx -= cx;
        by -= cy;
        bz -= cz;
        for (uint32_t o = T; o < 32u; o <<= 1) {
            bx += __shfl_xor_sync(0xFFFFFFFFu, bx, o);
            by += __shfl_xor_sync(0xFFFFFFFFu, by, o);
            bz += __shfl_xor_sync(0xFFFFFFFFu, bz, o);
        }
        if (active && slice == 0) {
            const float4 pp = part[tl];
            bx += pp.x;
            by += pp.y;
            bz += pp.z;
            const float4 L = tv.lt[u];
            float lx = L.y, ly = L.z, lz = L.w;
            if constexpr (GRAD) {
                const float4 cu = tv.geo[u];
                const float3 sh = grad_apply(tv.lg0[u], tv.lg1[u], t.x - cu.x, t.y - cu.y,
                                             t.z - cu.z);
                lx += sh.x;
                ly += sh.y;
                lz += sh.z;
                if (A.leaf_of) A.leaf_of[i] = u;
            }
            const double mm = (double)t.w;
            A.fx[i] = (float)(mm * ((double)lx + (double)bx));
            A.fy[i] = (float)(mm * ((double)ly + (double)by));
            A.fz[i] = (float)(mm * ((double)lz + (double)bz));
        }
        __syncwarp();
    }
    if (DEBUG) {
        inter = warp_sum(inter);
        if (lane == 0 && inter) {
            atomicAdd(&status->stat[PSG_STAT_P2P_INTER], inter);
            atomicAdd(&status->stat[PSG_STAT_DENSE_INTER], inter);
        }
    }
}

// L2L + L2P + P2P of the shallow leaves (depth <= heavy_depth; the leaf
// pass starts below them), one block each.  A shallow leaf is a large cell,
// so its walk -- the reference's (t leaf, s) recursion over the whole
// candidate set -- reaches a large part of the tree; the block runs it
// level-synchronously: the frontier of candidates at one level is tested by
// all threads (separated: M2L, leaf: P2P, else: its children go to the next
// frontier, placed by a block scan).
// Frontier order and the final reduction are fixed, so the result does not
// depend on scheduling.  A one-particle leaf sums its P2P during the walk; a
// leaf holding more (leaf capacity > 1) lists its P2P sources in frontier
// order and sums them per particle afterwards.
constexpr int kHeavyThreads = 512;
constexpr int kHeavyWarps = kHeavyThreads / 32;
constexpr int kHeavyTargets = 8;  // particles of a multi-particle leaf summed together

// exclusive block scan of v; returns the block total
__device__ __forceinline__ uint32_t block_scan(uint32_t v, uint32_t& excl, uint32_t* s_w) {
    const uint32_t lane = lane_id(), w = threadIdx.x >> 5;
    const uint32_t inc = warp_incl_scan(v);
    if (lane == 31) s_w[w] = inc;
    __syncthreads();
    uint32_t base = 0, total = 0;
    for (int k = 0; k < kHeavyWarps; ++k) {
        const uint32_t x = s_w[k];
        if (k < (int)w) base += x;
        total += x;
    }
    __syncthreads();
    excl = base + inc - v;
    return total;
}

template <bool DEBUG, bool GRAD>
__global__ void __launch_bounds__(kHeavyThreads, 2) k_heavy_leaf(TravArgs A) {
    __shared__ uint32_t s_w[kHeavyWarps];
    __shared__ uint32_t s_rec;
    __shared__ float s_red[kHeavyWarps][12];
    __shared__ float4 s_g[2];  // multi-particle leaf: field gradient (xx yy zz xy), local field
    __shared__ float2 s_g1;
    __shared__ unsigned long long s_cnt[kHeavyWarps][3];
    __shared__ float s_redt[kHeavyWarps][3 * kHeavyTargets];
    Status* status = A.status;
    // (a run whose near lists ran out is void: see k_trav)
    if (status->err & (PSG_ERR_NODES | PSG_ERR_SORT_SPIN | PSG_ERR_HEAVY_OVERFLOW |
                       PSG_ERR_NS_OVERFLOW))
        return;
    const TreeView& tv = A.tv;
    // work items: the leaf children of the nodes at depths 0 .. heavy_depth-1
    uint32_t cum[kMaxDepth + 1];
    uint32_t total = 0;
    for (int d = 0; d < A.heavy_depth && d < kMaxDepth; ++d) {
        cum[d] = total;
        total += status->lvl_count[d];
    }
    if (total == 0) return;
    const uint32_t tid = threadIdx.x, lane = lane_id(), w = tid >> 5;
    const float theta2 = __fmul_rn(A.theta, A.theta);
    uint32_t* fa = A.heavy_frontier + (size_t)blockIdx.x * 3 * A.heavy_fcap;
    uint32_t* fb = fa + A.heavy_fcap;
    uint32_t* const fp = fa + 2 * (size_t)A.heavy_fcap;  // P2P sources of a multi-particle leaf
    uint32_t leaves = 0, pid = 0, dp = 0, fc = 0;  // current group's leaf children
    uint32_t gsys = 0;                              // ... its system (batched systems)
    float th2 = theta2;
    for (;;) {
        if (leaves == 0) {
            // next group with leaf children
            if (tid == 0) s_rec = atomicAdd(&status->heavy_work, 1u);
            __syncthreads();
            const uint32_t g = s_rec;
            __syncthreads();
            if (g >= total) break;
            dp = 0;
            for (int d = 1; d < A.heavy_depth && d < kMaxDepth; ++d)
                if (g >= cum[d]) dp = d;
            pid = tv.lvl_base[dp] + (g - cum[dp]);
            if (tv.part_sys) {
                // batched systems: only the groups shallow for their own system
                gsys = tv.part_sys[tv.info[pid].x];
                if ((int)dp >= tv.sys_heavy[gsys]) continue;
                th2 = tv.sys_theta2[gsys];
            }
            const uint32_t plink = tv.link[pid];
            fc = plink & kLinkMask;
            for (uint32_t q = 0; q < (plink >> 28); ++q)
                if ((tv.link[fc + q] >> 28) == 0) leaves |= 1u << q;
            if (leaves == 0) continue;
        }
        const uint32_t u = fc + __ffs(leaves) - 1;
        leaves &= leaves - 1;
        const float4 ug = tv.geo[u];
        const uint4 ui = tv.info[u];
        const float4 t = A.xyzm[ui.x];
        const bool multi = ui.y > 1u;  // the same for the whole block
        uint32_t np2p = 0;
        // initial candidates: cand(p)
        uint32_t F = 0;
        if (dp <= 1) {
            if (tid == 0) fa[0] = gsys;  // the (system's) root
            F = 1;
        } else {
            const uint32_t* nsl = A.ns + tv.ns_off[pid];
            const uint32_t nsn = tv.ns_cnt[pid];
            for (uint32_t e0 = 0; e0 < nsn; e0 += kHeavyThreads) {
                const uint32_t e = e0 + tid;
                uint32_t s0 = 0, link = 0, c = 0;
                if (e < nsn) {
                    s0 = nsl[e];
                    link = tv.link[s0];
                    c = (link >> 28) ? (link >> 28) : 1u;
                }
                uint32_t ex;
                const uint32_t tot = block_scan(c, ex, s_w);
                if (F + tot > A.heavy_fcap) {
                    if (tid == 0) set_err(status, PSG_ERR_HEAVY_OVERFLOW);
                    return;
                }
                for (uint32_t i = 0; i < c; ++i)
                    fa[F + ex + i] = (link >> 28) ? (link & kLinkMask) + i : s0;
                F += tot;
            }
        }
        __syncthreads();
        float ax = 0.f, ay = 0.f, az = 0.f;
        float g[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        float bx = 0.f, by = 0.f, bz = 0.f, cx = 0.f, cy = 0.f, cz = 0.f;
        unsigned long long n_m2l = 0, n_p2p = 0, n_inter = 0;
        // one candidate: MAC, then M2L, a P2P source or its children
        auto visit = [&](uint32_t sn, float4 sg, uint32_t& c, uint32_t& link, uint32_t& pf) {
            float dx, dy, dz, d2;
            if (mac_separated(ug.x, ug.y, ug.z, ug.w, sg.x, sg.y, sg.z, sg.w, th2, dx, dy, dz,
                              d2)) {
                const float4 mp = tv.mp[sn];
                float fx, fy, fz;
                if constexpr (GRAD) {
                    float g3, gi;
                    m2l_field_grad(dx, dy, dz, d2, mp, fx, fy, fz, g3, gi);
                    g[0] += fmaf(g3 * dx, dx, -gi);
                    g[1] += fmaf(g3 * dy, dy, -gi);
                    g[2] += fmaf(g3 * dz, dz, -gi);
                    g[3] += g3 * dx * dy;
                    g[4] += g3 * dx * dz;
                    g[5] += g3 * dy * dz;
                } else {
                    m2l_field(dx, dy, dz, d2, mp, fx, fy, fz);
                }
                ax += fx;
                ay += fy;
                az += fz;
                ++n_m2l;
            } else {
                link = tv.link[sn];
                c = link >> 28;
                if (c == 0) {  // leaf x leaf: P2P
                    const uint4 si = tv.info[sn];
                    if (multi) {
                        pf = 1;
                    } else {
                        p2p_range(A.xyzm, make_uint2(si.x, si.y), t, A.kahan, bx, by, bz, cx, cy,
                                  cz);
                    }
                    ++n_p2p;
                    n_inter += (unsigned long long)si.y * ui.y;
                }
            }
        };
        while (F > 0) {
            uint32_t Fn = 0;
            // two candidates per thread and step (candidates i and i + 512 of
            // the step's 1024), their loads in flight together; one block
            // scan places both threads' children and P2P sources
            for (uint32_t i0 = 0; i0 < F; i0 += 2 * kHeavyThreads) {
                const uint32_t ia = i0 + tid, ib = ia + kHeavyThreads;
                const uint32_t sa = ia < F ? fa[ia] : kNone, sb = ib < F ? fa[ib] : kNone;
                const float4 ga = sa != kNone ? tv.geo[sa] : make_float4(0.f, 0.f, 0.f, 0.f);
                const float4 gb = sb != kNone ? tv.geo[sb] : make_float4(0.f, 0.f, 0.f, 0.f);
                uint32_t ca = 0, la = 0, pa = 0, cb = 0, lb = 0, pb = 0;
                if (sa != kNone) visit(sa, ga, ca, la, pa);
                if (sb != kNone) visit(sb, gb, cb, lb, pb);
                // children counts in bits 0..15 (at most 8 x 1024 a step), P2P
                // sources above
                uint32_t ex;
                const uint32_t tot = block_scan((ca + cb) | ((pa + pb) << 16), ex, s_w);
                const uint32_t ctot = tot & 0xFFFFu, ptot = tot >> 16;
                const uint32_t cex = ex & 0xFFFFu, pex = ex >> 16;
                if (Fn + ctot > A.heavy_fcap || np2p + ptot > A.heavy_fcap) {
                    if (tid == 0) set_err(status, PSG_ERR_HEAVY_OVERFLOW);
                    return;
                }
                if (pa) fp[np2p + pex] = sa;
                if (pb) fp[np2p + pex + pa] = sb;
                np2p += ptot;
                for (uint32_t k = 0; k < ca; ++k) fb[Fn + cex + k] = (la & kLinkMask) + k;
                for (uint32_t k = 0; k < cb; ++k) fb[Fn + cex + ca + k] = (lb & kLinkMask) + k;
                Fn += ctot;
            }
            __syncthreads();
            uint32_t* tmp = fa;
            fa = fb;
            fb = tmp;
            F = Fn;
        }
        // fixed-order block reduction
        float v[12] = {ax, ay, az, g[0], g[1], g[2], g[3], g[4], g[5], bx - cx, by - cy, bz - cz};
#pragma unroll
        for (int k = 0; k < 12; ++k) {
            const float x = warp_sum(v[k]);
            if (lane == 0) s_red[w][k] = x;
        }
        if (DEBUG) {
            const unsigned long long c0 = warp_sum(n_m2l), c1 = warp_sum(n_p2p),
                                     c2 = warp_sum(n_inter);
            if (lane == 0) {
                s_cnt[w][0] = c0;
                s_cnt[w][1] = c1;
                s_cnt[w][2] = c2;
            }
        }
        __syncthreads();
        if (tid == 0) {
            float sum[12];
            for (int k = 0; k < 12; ++k) {
                sum[k] = 0.f;
                for (int q = 0; q < kHeavyWarps; ++q) sum[k] += s_red[q][k];
            }
            // L2L from the parent, then L2P at the particle
            const float4 Lp = tv.lt[pid];
            float4 L = make_float4(0.f, __fadd_rn(sum[0], Lp.y), __fadd_rn(sum[1], Lp.z),
                                   __fadd_rn(sum[2], Lp.w));
            float lx = L.y, ly = L.z, lz = L.w;
            if constexpr (GRAD) {
                float4 G0 = make_float4(sum[3], sum[4], sum[5], sum[6]);
                float2 G1 = make_float2(sum[7], sum[8]);
                if (dp >= 2) {
                    const float4 cp = tv.geo[pid];
                    const float4 Gp0 = tv.lg0[pid];
                    const float2 Gp1 = tv.lg1[pid];
                    const float3 sh = grad_apply(Gp0, Gp1, ug.x - cp.x, ug.y - cp.y, ug.z - cp.z);
                    L.y += sh.x;
                    L.z += sh.y;
                    L.w += sh.z;
                    G0.x += Gp0.x;
                    G0.y += Gp0.y;
                    G0.z += Gp0.z;
                    G0.w += Gp0.w;
                    G1.x += Gp1.x;
                    G1.y += Gp1.y;
                }
                tv.lg0[u] = G0;
                tv.lg1[u] = G1;
                s_g[0] = G0;
                s_g1 = G1;
                const float3 at = grad_apply(G0, G1, t.x - ug.x, t.y - ug.y, t.z - ug.z);
                lx = L.y + at.x;
                ly = L.z + at.y;
                lz = L.w + at.z;
                if (A.leaf_of && !multi) A.leaf_of[ui.x] = u;
            }
            tv.lt[u] = L;
            s_g[1] = L;
            if (!multi) {
                const double mm = (double)t.w;
                A.fx[ui.x] = (float)(mm * ((double)lx + (double)sum[9]));
                A.fy[ui.x] = (float)(mm * ((double)ly + (double)sum[10]));
                A.fz[ui.x] = (float)(mm * ((double)lz + (double)sum[11]));
            }
            if (DEBUG) {
                unsigned long long c0 = 0, c1 = 0, c2 = 0;
                for (int q = 0; q < kHeavyWarps; ++q) {
                    c0 += s_cnt[q][0];
                    c1 += s_cnt[q][1];
                    c2 += s_cnt[q][2];
                }
                tv.dbg_m2l[u] = (uint32_t)c0;
                tv.dbg_p2p[u] = (uint32_t)c1;
                atomicAdd(&status->stat[PSG_STAT_M2L], c0);
                atomicAdd(&status->stat[PSG_STAT_P2P_PAIRS], c1);
                atomicAdd(&status->stat[PSG_STAT_P2P_INTER], c2);
            }
        }
        __syncthreads();
        if (multi) {
            // P2P + L2P of the leaf's particles over the listed sources,
            // kHeavyTargets particles a pass: each source particle is loaded
            // once a pass and summed into every target's accumulators;
            // fixed-order sums over warps, then over the block
            const float4 L = s_g[1];
            for (uint32_t k0 = 0; k0 < ui.y; k0 += kHeavyTargets) {
                const uint32_t nk = min((uint32_t)kHeavyTargets, ui.y - k0);
                float4 tk[kHeavyTargets];
                float acc[kHeavyTargets][3];
#pragma unroll
                for (int k = 0; k < kHeavyTargets; ++k) {
                    tk[k] = A.xyzm[ui.x + k0 + min((uint32_t)k, nk - 1)];
                    acc[k][0] = acc[k][1] = acc[k][2] = 0.f;
                }
                if (A.kahan) {
                    // compensated sums: one target at a time (a rare mode)
                    for (uint32_t k = 0; k < nk; ++k) {
                        float px = 0.f, py = 0.f, pz = 0.f, qx = 0.f, qy = 0.f, qz = 0.f;
                        const float4 t1 = A.xyzm[ui.x + k0 + k];
                        for (uint32_t e = tid; e < np2p; e += kHeavyThreads) {
                            const uint4 si = tv.info[fp[e]];
                            p2p_range(A.xyzm, make_uint2(si.x, si.y), t1, true, px, py, pz, qx,
                                      qy, qz);
                        }
#pragma unroll
                        for (int kk = 0; kk < kHeavyTargets; ++kk)
                            if ((uint32_t)kk == k) {
                                acc[kk][0] = px - qx;
                                acc[kk][1] = py - qy;
                                acc[kk][2] = pz - qz;
                            }
                    }
                } else {
                    // the listed source leaves, 32 a warp at a time, their
                    // particles laid end to end (a warp prefix sum) and dealt
                    // one per lane, so that no lane idles on a short leaf;
                    // the targets two at a time in paired FP32 instructions
                    constexpr int KP = kHeavyTargets / 2;
                    float2 ntx[KP], nty[KP], ntz[KP], sx[KP], sy[KP], sz[KP];
#pragma unroll
                    for (int k = 0; k < KP; ++k) {
                        ntx[k] = make_float2(-tk[2 * k].x, -tk[2 * k + 1].x);
                        nty[k] = make_float2(-tk[2 * k].y, -tk[2 * k + 1].y);
                        ntz[k] = make_float2(-tk[2 * k].z, -tk[2 * k + 1].z);
                        sx[k] = sy[k] = sz[k] = make_float2(0.f, 0.f);
                    }
                    const float2 eps = make_float2(0.1f, 0.1f);
                    for (uint32_t e0 = w * 32u; e0 < np2p; e0 += kHeavyThreads) {
                        uint32_t es = 0, en = 0;
                        if (e0 + lane < np2p) {
                            const uint4 si = tv.info[fp[e0 + lane]];
                            es = si.x;
                            en = si.y;
                        }
                        const uint32_t incl = warp_incl_scan(en);
                        const uint32_t ptot = __shfl_sync(0xFFFFFFFFu, incl, 31);
                        const uint32_t excl = incl - en;
                        for (uint32_t b = 0; b < ptot; b += 32) {
                            // lane's particle: the entry whose prefix holds b + lane
                            const uint32_t f = b + lane;
                            uint32_t ee = 0;
#pragma unroll
                            for (uint32_t step = 16; step > 0; step >>= 1) {
                                const uint32_t v = __shfl_sync(0xFFFFFFFFu, incl, ee + step - 1);
                                if (v <= f) ee += step;
                            }
                            const uint32_t s0 = __shfl_sync(0xFFFFFFFFu, es, ee);
                            const uint32_t x0 = __shfl_sync(0xFFFFFFFFu, excl, ee);
                            if (f < ptot) {
                                const float4 p = A.xyzm[s0 + (f - x0)];
                                const float2 px = make_float2(p.x, p.x), py = make_float2(p.y, p.y),
                                             pz = make_float2(p.z, p.z), pw = make_float2(p.w, p.w);
#pragma unroll
                                for (int k = 0; k < KP; ++k) {
                                    const float2 dx = __fadd2_rn(px, ntx[k]);
                                    const float2 dy = __fadd2_rn(py, nty[k]);
                                    const float2 dz = __fadd2_rn(pz, ntz[k]);
                                    float2 r = __ffma2_rn(dz, dz, eps);
                                    r = __ffma2_rn(dy, dy, r);
                                    r = __ffma2_rn(dx, dx, r);
                                    const float2 i = make_float2(rsqrtf(r.x), rsqrtf(r.y));
                                    const float2 fw =
                                        __fmul2_rn(pw, __fmul2_rn(__fmul2_rn(i, i), i));
                                    sx[k] = __ffma2_rn(dx, fw, sx[k]);
                                    sy[k] = __ffma2_rn(dy, fw, sy[k]);
                                    sz[k] = __ffma2_rn(dz, fw, sz[k]);
                                }
                            }
                        }
                    }
#pragma unroll
                    for (int k = 0; k < KP; ++k) {
                        acc[2 * k][0] = sx[k].x;
                        acc[2 * k + 1][0] = sx[k].y;
                        acc[2 * k][1] = sy[k].x;
                        acc[2 * k + 1][1] = sy[k].y;
                        acc[2 * k][2] = sz[k].x;
                        acc[2 * k + 1][2] = sz[k].y;
                    }
                }
#pragma unroll
                for (int k = 0; k < kHeavyTargets; ++k) {
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        const float x = warp_sum(acc[k][c]);
                        if (lane == 0) s_redt[w][3 * k + c] = x;
                    }
                }
                __syncthreads();
                if (tid < nk) {
                    float sx = 0.f, sy = 0.f, sz = 0.f;
                    for (int q = 0; q < kHeavyWarps; ++q) {
                        sx += s_redt[q][3 * tid];
                        sy += s_redt[q][3 * tid + 1];
                        sz += s_redt[q][3 * tid + 2];
                    }
                    const uint32_t i = ui.x + k0 + tid;
                    const float4 t1 = A.xyzm[i];
                    float lx = L.y, ly = L.z, lz = L.w;
                    if constexpr (GRAD) {
                        const float3 at =
                            grad_apply(s_g[0], s_g1, t1.x - ug.x, t1.y - ug.y, t1.z - ug.z);
                        lx += at.x;
                        ly += at.y;
                        lz += at.z;
                        if (A.leaf_of) A.leaf_of[i] = u;
                    }
                    const double mm = (double)t1.w;
                    A.fx[i] = (float)(mm * ((double)lx + (double)sx));
                    A.fy[i] = (float)(mm * ((double)ly + (double)sy));
                    A.fz[i] = (float)(mm * ((double)lz + (double)sz));
                }
                __syncthreads();
            }
        }
    }
}

// the leaf pass's work counter starts past the groups of depths 0 ..
// heavy_depth-1, whose leaf children k_heavy_leaf takes
__global__ void k_leaf_start(Status* status, int heavy_depth, uint32_t parts) {
    uint32_t skip = 0;
    for (int d = 0; d < heavy_depth && d < kMaxDepth; ++d) skip += status->lvl_count[d];
    status->work[0] = skip * parts;
}

void launch_leaf_start(Status* status, int heavy_depth, int order, cudaStream_t st) {
    // work items per group: 2 halves with the order-1 accumulators, else 1
    k_leaf_start<<<1, 1, 0, st>>>(status, heavy_depth, order >= 1 ? 2u : 1u);
}

void launch_heavy_leaf(const TravArgs& A, int grid, cudaStream_t st) {
    if (A.order >= 1) {
        if (A.debug) k_heavy_leaf<true, true><<<grid, kHeavyThreads, 0, st>>>(A);
        else k_heavy_leaf<false, true><<<grid, kHeavyThreads, 0, st>>>(A);
    } else {
        if (A.debug) k_heavy_leaf<true, false><<<grid, kHeavyThreads, 0, st>>>(A);
        else k_heavy_leaf<false, false><<<grid, kHeavyThreads, 0, st>>>(A);
    }
}

template <bool DEBUG, bool GRAD>
static void launch_dense_kahan(const TravArgs& A, int grid, cudaStream_t st) {
    if (A.kahan) k_dense_p2p<DEBUG, GRAD, true><<<grid, kTravThreads, 0, st>>>(A);
    else k_dense_p2p<DEBUG, GRAD, false><<<grid, kTravThreads, 0, st>>>(A);
}

void launch_dense_p2p(const TravArgs& A, int grid, cudaStream_t st) {
    if (A.order >= 1) {
        if (A.debug) launch_dense_kahan<true, true>(A, grid, st);
        else launch_dense_kahan<false, true>(A, grid, st);
    } else {
        if (A.debug) launch_dense_kahan<true, false>(A, grid, st);
        else launch_dense_kahan<false, false>(A, grid, st);
    }
}

template <int MODE, bool DENSE, bool XL>
static void launch_mode(const TravArgs& A, int grid, cudaStream_t st) {
    if (A.order >= 1) {
        if (A.debug) k_trav<MODE, true, true, DENSE, XL><<<grid, kTravThreads, 0, st>>>(A);
        else k_trav<MODE, false, true, DENSE, XL><<<grid, kTravThreads, 0, st>>>(A);
    } else {
        if (A.debug) k_trav<MODE, true, false, DENSE, XL><<<grid, kTravThreads, 0, st>>>(A);
        else k_trav<MODE, false, false, DENSE, XL><<<grid, kTravThreads, 0, st>>>(A);
    }
}

static bool leaf_xl(const TravArgs& A) { return A.ns_levels < kMaxDepth || A.stream; }

void launch_traverse_internal(const TravArgs& args, int level, int grid, cudaStream_t st) {
    TravArgs A = args;
    A.level = level;
    launch_mode<MODE_INTERNAL, false, false>(A, grid, st);
}

void launch_traverse_leaves(const TravArgs& args, const int grid[2], cudaStream_t st) {
    if (leaf_xl(args)) {
        launch_mode<MODE_LEAF, false, true>(args, grid[0], st);
        launch_mode<MODE_LEAF, true, true>(args, grid[1], st);
    } else {
        launch_mode<MODE_LEAF, false, false>(args, grid[0], st);
        launch_mode<MODE_LEAF, true, false>(args, grid[1], st);
    }
}

int traverse_threads() { return kTravThreads; }
const void* traverse_kernel_ptr(int order, int dense, int xl) {
    if (xl) {
        if (order) {
            return dense ? (const void*)k_trav<MODE_LEAF, false, true, true, true>
                         : (const void*)k_trav<MODE_LEAF, false, true, false, true>;
        }
        return dense ? (const void*)k_trav<MODE_LEAF, false, false, true, true>
                     : (const void*)k_trav<MODE_LEAF, false, false, false, true>;
    }
    if (order) {
        return dense ? (const void*)k_trav<MODE_LEAF, false, true, true, false>
                     : (const void*)k_trav<MODE_LEAF, false, true, false, false>;
    }
    return dense ? (const void*)k_trav<MODE_LEAF, false, false, true, false>
                 : (const void*)k_trav<MODE_LEAF, false, false, false, false>;
}
const void* traverse_internal_kernel_ptr(int order) {
    return order ? (const void*)k_trav<MODE_INTERNAL, false, true, false, false>
                 : (const void*)k_trav<MODE_INTERNAL, false, false, false, false>;
}

}  // namespace psg
