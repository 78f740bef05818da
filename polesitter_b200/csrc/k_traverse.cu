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
// the sources it was not separated from, so every child u of an internal
// node p starts from the same candidates
//   cand(p) = {root}                                         if depth(p) <= 1
//   cand(p) = U_{s in NS(p)} (s leaf ? {s} : children(s))    otherwise.
// One warp owns a parent p and takes its target children one after the
// other; for a child u the lanes test 32 candidates at a time with the MAC,
// accumulate M2L in registers, and deal with the near ones:
//
//  * MODE_INTERNAL, one launch per level k = 2..10, targets = the internal
//    children of the depth-(k-1) nodes: near candidates form NS(u) in HBM for
//    level k+1, and L(u) = M2L(u) + L(p) is stored.
//  * MODE_LEAF, one launch after all levels, targets = the leaf children of
//    every node: a near leaf candidate is a P2P source (staged in shared
//    memory, spilled to HBM chunks only past 32), a near internal candidate
//    is the "t leaf" recursion and goes onto a DFS stack in shared memory
//    that is drained the same way.  The warp then finishes u:
//    L(u) = M2L(u) + L(p) and, per particle, F = m * (L(u) + its P2P sum) --
//    written once, no atomics.  Running all levels' leaves in one launch lets
//    the long descents of shallow leaves overlap with everything else.
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
constexpr int kCandBuf = 256;             // children of 32 opened entries
constexpr int kStackCap = 384;            // DFS stack (node ids)
constexpr int kStackSlack = 72;           // 9 levels x 7: growth of a single-entry descent
constexpr uint32_t kNsPool = 4096;        // near-list entries a warp reserves at once
constexpr uint32_t kChunkPool = 16;       // P2P spill chunks a warp reserves at once

enum { MODE_INTERNAL = 0, MODE_LEAF = 1 };

struct SmemInternal {
    float4 cgeo[8];  // the parent's children: centre + half width
    uint32_t cand[kCandBuf];
    unsigned long long ns_next, ns_end;
};

struct SmemLeaf {
    float4 cgeo[8];
    uint32_t cand[kCandBuf];
    uint32_t stk[kStackCap];
    uint32_t p2p[kP2PChunk];
    uint32_t chunk_next, chunk_end;
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

// Spill the staged P2P sources of the current leaf as one chunk chained to
// its previous one.  Warp-collective; chunk ids come from a per-warp pool.
__device__ __noinline__ uint32_t spill_p2p(SmemLeaf& sm, uint32_t fill, uint32_t head,
                                           P2PStore st, Status* status) {
    const uint32_t lane = lane_id();
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
    const bool ok = c < st.cap_chunks;
    if (ok) {
        if (lane < fill) st.src[(size_t)c * kP2PChunk + lane] = sm.p2p[lane];
        if (lane == 0) {
            st.next[c] = head;
            st.cnt[c] = fill;
        }
    } else if (lane == 0) {
        set_err(status, PSG_ERR_P2P_OVERFLOW);
    }
    __syncwarp();
    if (lane == 0) sm.chunk_next = c + 1;
    __syncwarp();
    return ok ? c : head;
}

// Direct sum of the particles of source leaf si on target particle t
// (polesitter.h:1424-1444 with rsqrt), optionally Kahan-compensated.
__device__ __forceinline__ void p2p_leaf(const float4* __restrict__ xyzm, uint4 si, float4 t,
                                         bool kahan, float& ax, float& ay, float& az, float& cx,
                                         float& cy, float& cz) {
    for (uint32_t j = 0; j < si.y; ++j) {
        const float4 p = xyzm[si.x + j];
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

template <int MODE, bool DEBUG>
__global__ void __launch_bounds__(kTravThreads) k_trav(TravArgs A) {
    using Smem = typename SmemOf<MODE>::T;
    __shared__ Smem smem[kTravWarps];
    const uint32_t lane = lane_id();
    const uint32_t lt_mask = lanemask_lt();
    Smem& sm = smem[threadIdx.x >> 5];
    const TreeView& tv = A.tv;
    Status* status = A.status;
    if (status->err & (PSG_ERR_NODES | PSG_ERR_SORT_SPIN)) return;
    const float theta2 = __fmul_rn(A.theta, A.theta);

    // parent index space: MODE_INTERNAL = the nodes at depth k-1; MODE_LEAF =
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
        work = &status->work[0];
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
    const uint32_t batch = MODE == MODE_INTERNAL ? 4u : 8u;

    for (;;) {
        uint32_t g0 = 0;
        if (lane == 0) g0 = atomicAdd(work, batch);
        g0 = __shfl_sync(0xFFFFFFFFu, g0, 0);
        if (g0 >= total) break;
#pragma unroll 1
        for (uint32_t g = g0; g < g0 + batch && g < total; ++g) {
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
            const uint32_t plink = tv.link[pid];
            const uint32_t nc = plink >> 28;
            if (nc == 0) continue;
            const uint32_t fc = plink & kLinkMask;
            uint32_t cl = 0;
            if (lane < nc) {
                sm.cgeo[lane] = tv.geo[fc + lane];
                cl = tv.link[fc + lane];
            }
            const uint32_t leaf_mask =
                __ballot_sync(0xFFFFFFFFu, lane < nc && (cl >> 28) == 0) & 0xFFu;
            const uint32_t tgt_mask =
                MODE == MODE_INTERNAL ? (((1u << nc) - 1u) & ~leaf_mask) : leaf_mask;
            if (tgt_mask == 0) continue;
            const float4 Lp = tv.lt[pid];
            const bool root_only = dp <= 1;
            const uint32_t* nsl = nullptr;
            uint32_t nsn = 0;
            if (!root_only) {
                nsl = A.ns + tv.ns_off[pid];
                nsn = tv.ns_cnt[pid];
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
                if (!ns_ok && lane == 0) set_err(status, PSG_ERR_NS_OVERFLOW);
                __syncwarp();
                if (lane == 0) sm.ns_next = ns_base + need;
                __syncwarp();
            }

            uint32_t sub = 0;  // rank of the target child among the targets
#pragma unroll 1
            for (uint32_t tm = tgt_mask; tm; tm &= tm - 1, ++sub) {
                const uint32_t q = __ffs(tm) - 1;
                const uint32_t u = fc + q;
                const float4 ug = sm.cgeo[q];
                float ax = 0.f, ay = 0.f, az = 0.f;
                uint32_t n_near = 0;   // MODE_INTERNAL: entries of NS(u)
                uint32_t fill = 0;     // MODE_LEAF: staged P2P sources
                uint32_t head = kNone; // MODE_LEAF: last spilled chunk
                uint32_t dbg_m2l = 0, dbg_p2p = 0;
                uint32_t ssize = 0, e0 = 0;
                bool root_pending = root_only;
                for (;;) {
                    // ---- next batch of candidates into cand[0, tot) ----
                    uint32_t tot;
                    if (root_pending) {
                        if (lane == 0) sm.cand[0] = 0;  // the root
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
                        for (uint32_t i = 0; i < c; ++i)
                            sm.cand[ex + i] = lf ? s0 : (link & kLinkMask) + i;
                        e0 += 32;
                    } else if (MODE == MODE_LEAF && ssize > 0) {
                        // pop entries (bounded so the stack cannot overflow), open them
                        const int room = ((int)kStackCap - kStackSlack - (int)ssize) / 7;
                        const uint32_t kp = (uint32_t)min(32, min((int)ssize, max(1, room)));
                        uint32_t node = 0;
                        if constexpr (MODE == MODE_LEAF) {
                            if (lane < kp) node = sm.stk[ssize - kp + lane];
                        }
                        __syncwarp();
                        ssize -= kp;
                        const uint32_t link = lane < kp ? tv.link[node] : 0u;
                        const uint32_t nch = link >> 28;
                        const uint32_t inc = warp_incl_scan(nch);
                        tot = __shfl_sync(0xFFFFFFFFu, inc, 31);
                        const uint32_t ex = inc - nch;
                        for (uint32_t i = 0; i < nch; ++i) sm.cand[ex + i] = (link & kLinkMask) + i;
                    } else {
                        break;
                    }
                    __syncwarp();

                    // ---- test the candidates, one per lane ----
#pragma unroll 1
                    for (uint32_t j0 = 0; j0 < tot; j0 += 32) {
                        const uint32_t j = j0 + lane;
                        const bool valid = j < tot;
                        uint32_t s = 0, slink = 0;
                        float4 sg = make_float4(0.f, 0.f, 0.f, 0.f), smp = sg;
                        if (valid) {
                            s = sm.cand[j];
                            sg = tv.geo[s];
                            smp = tv.mp[s];
                            slink = tv.link[s];
                        }
                        float dx, dy, dz, d2;
                        const bool sep = mac_separated(ug.x, ug.y, ug.z, ug.w, sg.x, sg.y, sg.z,
                                                       sg.w, theta2, dx, dy, dz, d2) && valid;
                        if (sep) {
                            float fx, fy, fz;
                            m2l_field(dx, dy, dz, d2, smp, fx, fy, fz);
                            ax += fx;
                            ay += fy;
                            az += fz;
                        }
                        if (DEBUG) dbg_m2l += __popc(__ballot_sync(0xFFFFFFFFu, sep));
                        const bool near = valid && !sep;
                        if constexpr (MODE == MODE_INTERNAL) {
                            const uint32_t nm = __ballot_sync(0xFFFFFFFFu, near);
                            if (near && ns_ok)
                                A.ns[ns_base + (unsigned long long)sub * cand_total + n_near +
                                     __popc(nm & lt_mask)] = s;
                            n_near += __popc(nm);
                        } else {
                            const bool sleaf = (slink >> 28) == 0;
                            // near leaf: P2P source
                            uint32_t pm = __ballot_sync(0xFFFFFFFFu, near && sleaf);
                            if (DEBUG) dbg_p2p += __popc(pm);
                            while (pm) {
                                if (fill == (uint32_t)kP2PChunk) {
                                    head = spill_p2p(sm, fill, head, A.p2p, status);
                                    fill = 0;
                                }
                                const uint32_t space = kP2PChunk - fill;
                                const uint32_t rank = __popc(pm & lt_mask);
                                const bool take = ((pm >> lane) & 1u) && rank < space;
                                if (take) sm.p2p[fill + rank] = s;
                                const uint32_t taken = __ballot_sync(0xFFFFFFFFu, take);
                                pm &= ~taken;
                                fill += __popc(taken);
                                __syncwarp();
                            }
                            // near internal source: open it later (the "t leaf" recursion)
                            const bool push = near && !sleaf;
                            const uint32_t qm = __ballot_sync(0xFFFFFFFFu, push);
                            if (qm) {
                                const uint32_t pos = ssize + __popc(qm & lt_mask);
                                if (push && pos < (uint32_t)kStackCap) sm.stk[pos] = s;
                                ssize += __popc(qm);
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

                // ---- L2L; for leaves L2P + P2P ----
                ax = warp_sum(ax);
                ay = warp_sum(ay);
                az = warp_sum(az);
                // L(u) = M2L(u) + L(parent)  (polesitter.h:1248-1250)
                const float4 L = make_float4(0.f, __fadd_rn(ax, Lp.y), __fadd_rn(ay, Lp.z),
                                             __fadd_rn(az, Lp.w));
                if (lane == 0) tv.lt[u] = L;
                if constexpr (MODE == MODE_INTERNAL) {
                    if (lane == 0) {
                        tv.ns_off[u] = (uint32_t)(ns_base + (unsigned long long)sub * cand_total);
                        tv.ns_cnt[u] = ns_ok ? n_near : 0u;
                    }
                } else {
                    // P2P sources: the staged ones (lane < fill) and spilled chunks
                    const uint4 ui = tv.info[u];
                    uint4 si0 = make_uint4(0, 0, 0, 0);
                    if (lane < fill) si0 = tv.info[sm.p2p[lane]];
                    unsigned long long inter = 0;
                    for (uint32_t ti = 0; ti < ui.y; ++ti) {
                        const float4 t = A.xyzm[ui.x + ti];
                        float bx = 0.f, by = 0.f, bz = 0.f, cx = 0.f, cy = 0.f, cz = 0.f;
                        p2p_leaf(A.xyzm, si0, t, A.kahan, bx, by, bz, cx, cy, cz);
                        if (DEBUG) inter += si0.y;
                        for (uint32_t c = head; c != kNone; c = A.p2p.next[c]) {
                            if (lane < A.p2p.cnt[c]) {
                                const uint4 si = tv.info[A.p2p.src[(size_t)c * kP2PChunk + lane]];
                                p2p_leaf(A.xyzm, si, t, A.kahan, bx, by, bz, cx, cy, cz);
                                if (DEBUG) inter += si.y;
                            }
                        }
                        // lane partials (compensated) summed in FP64
                        const double sx = warp_sum((double)bx - (double)cx);
                        const double sy = warp_sum((double)by - (double)cy);
                        const double sz = warp_sum((double)bz - (double)cz);
                        if (lane == 0) {
                            const size_t gi = (size_t)ui.x + ti;
                            const double mm = (double)t.w;
                            A.fx[gi] = (float)(mm * ((double)L.y + sx));
                            A.fy[gi] = (float)(mm * ((double)L.z + sy));
                            A.fz[gi] = (float)(mm * ((double)L.w + sz));
                        }
                    }
                    if (DEBUG) {
                        inter = warp_sum(inter);
                        if (lane == 0) {
                            tv.dbg_p2p[u] = dbg_p2p;
                            atomicAdd(&status->stat[PSG_STAT_P2P_PAIRS], (unsigned long long)dbg_p2p);
                            atomicAdd(&status->stat[PSG_STAT_P2P_INTER], inter);
                        }
                    }
                    __syncwarp();
                }
                if (DEBUG && lane == 0) {
                    tv.dbg_m2l[u] = dbg_m2l;
                    atomicAdd(&status->stat[PSG_STAT_M2L], (unsigned long long)dbg_m2l);
                }
            }
            __syncwarp();
        }
    }
}

void launch_traverse_internal(const TravArgs& args, int level, int grid, cudaStream_t st) {
    TravArgs A = args;
    A.level = level;
    if (A.debug) k_trav<MODE_INTERNAL, true><<<grid, kTravThreads, 0, st>>>(A);
    else k_trav<MODE_INTERNAL, false><<<grid, kTravThreads, 0, st>>>(A);
}

void launch_traverse_leaves(const TravArgs& args, int grid, cudaStream_t st) {
    if (args.debug) k_trav<MODE_LEAF, true><<<grid, kTravThreads, 0, st>>>(args);
    else k_trav<MODE_LEAF, false><<<grid, kTravThreads, 0, st>>>(args);
}

int traverse_threads() { return kTravThreads; }
const void* traverse_kernel_ptr() { return (const void*)k_trav<MODE_LEAF, false>; }
const void* traverse_internal_kernel_ptr() { return (const void*)k_trav<MODE_INTERNAL, false>; }

}  // namespace psg
