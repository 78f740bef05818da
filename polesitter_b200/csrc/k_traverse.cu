// The interaction pass of the FMM tick, fused: MAC + M2L + L2L + L2P + P2P.
//
// Reference (PS_MULTITHREADING build): every node at depth 2, and every leaf
// above it, is paired with the root (ps_impl_dispatch_fmm, polesitter.h:
// 1772-1801, :1883-1885), and each pair (t, s) is walked by the dual
// recursion of ps_impl_fmm_interaction_pass (:1050-1146):
//   separated (MAC)        -> M2L: t.local += field of s's monopole+dipole
//   both leaves            -> left to P2P (the P2P pass :1258-1494 walks the
//                             same pairs with the same MAC)
//   t leaf                 -> (t, each child of s)
//   s leaf                 -> (each child of t, s)
//   otherwise              -> (each child of t) x (each child of s)
// then L2L adds every parent's field to its children (:1238-1251) and L2P
// gives F = m * field at the leaves (:1224-1233), then P2P adds the direct
// leaf x leaf sums.
//
// B200 formulation (target-major, level-synchronous, no pair lists in HBM):
// every pair (t, s) the recursion visits with an internal t at depth k and
// internal s has its children pairs generated from t's "near list" NS(t) =
// the sources s that t was not separated from.  So for each internal node p
// at depth k-1 ("group"), the candidates of ALL its children are
//   cand(p) = {root}                                  if k <= 2
//   cand(p) = U_{s in NS(p)} (s leaf ? {s} : children(s))   otherwise
// and one warp processes a group: lane j holds candidate j's centre,
// multipole and links in registers and tests it against every child u of p
// (<= 8), accumulating M2L in registers.  Non-separated candidates go to
// NS(u) when u is internal (written to HBM for level k+1), to u's P2P buffer
// when both are leaves, and onto a bounded DFS stack in shared memory when u
// is a leaf and s is internal (the "t leaf" recursion).  A leaf's visits all
// happen inside this warp, so the warp also finishes it: L(u) = M2L(u) +
// L(p) (L2L), and F_i = m_i * (L(u) + sum of P2P) for its particles, written
// once, with no atomics.  Internal children get L(u) = M2L(u) + L(p) stored
// for their own groups at level k+1.
//
// The MAC replays the reference's rounded float sequence exactly
// (mac_separated), so the interaction set is identical, ties included.
// Bound: FP32 pipe (M2L ~35 flop + 1 MUFU per pair, P2P ~20 flop + 1 MUFU).
#include "psg_common.cuh"
#include "psg_kernels.h"

namespace psg {

constexpr int kTravWarps = 4;
constexpr int kTravThreads = kTravWarps * 32;
constexpr int kCandBuf = 256;     // one expanded chunk of 32 near-list entries
constexpr int kStackCap = 512;    // DFS stack (entries: slot << 28 | node)
constexpr int kStackSlack = 72;   // 9 levels x 7 growth of a single-entry descent
constexpr int kP2PBuf = 128;      // buffered P2P source leaves (slot << 28 | node)
constexpr uint32_t kNodeMask = (1u << 28) - 1;
constexpr int kGroupBatch = 4;

struct TravArgs {
    TreeView tv;
    const float4* xyzm;
    float* fx;
    float* fy;
    float* fz;
    const uint32_t* ns_in;
    uint32_t* ns_out;
    unsigned long long ns_cap;
    double* facc;          // [N][3] partial P2P sums for multi-flush leaves
    Status* status;
    float theta;
    int level;
    int debug;
};

struct WarpSmem {
    float4 cgeo[8];
    uint4 cinfo[8];
    uint32_t cand[kCandBuf];
    uint32_t stk[kStackCap];
    uint32_t p2p[kP2PBuf];
};

struct M2LAcc {
    float v[8][3];
};

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
    const float b = ir3;
    fx = fmaf(dx, a, mp.y * b);
    fy = fmaf(dy, a, mp.z * b);
    fz = fmaf(dz, a, mp.w * b);
}

__device__ __forceinline__ void acc_add_dyn(M2LAcc& acc, uint32_t slot, float fx, float fy,
                                            float fz) {
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        if ((uint32_t)q == slot) {
            acc.v[q][0] += fx;
            acc.v[q][1] += fy;
            acc.v[q][2] += fz;
        }
    }
}

// Direct sums of the buffered P2P pairs (polesitter.h:1279-1449 with rsqrt):
// for every leaf target slot and each of its particles, lanes walk the
// buffered source leaves of that slot; the warp total goes to facc (or, on
// the last flush, into the returned per-particle value via `fin`).
__device__ void p2p_flush(const TravArgs& A, WarpSmem& sm, uint32_t np, uint32_t leaf_slots,
                          bool last, bool& flushed_before, const float4* Lslot) {
    const uint32_t lane = lane_id();
    const TreeView& tv = A.tv;
#pragma unroll 1
    for (uint32_t sl = 0; sl < 8; ++sl) {
        if (!((leaf_slots >> sl) & 1u)) continue;
        const uint4 ui = sm.cinfo[sl];
        const uint32_t ustart = ui.x, ucnt = ui.y;
#pragma unroll 1
        for (uint32_t ti = 0; ti < ucnt; ++ti) {
            const float4 t = A.xyzm[ustart + ti];
            float ax = 0.f, ay = 0.f, az = 0.f;
            for (uint32_t e = lane; e < np; e += 32) {
                const uint32_t ent = sm.p2p[e];
                if ((ent >> 28) != sl) continue;
                const uint4 si = tv.info[ent & kNodeMask];
                for (uint32_t j = 0; j < si.y; ++j) {
                    const float4 p = A.xyzm[si.x + j];
                    const float dx = p.x - t.x, dy = p.y - t.y, dz = p.z - t.z;
                    const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz)) + 0.1f;
                    const float inv = rsqrtf(r2);
                    const float f = p.w * (inv * inv * inv);
                    ax = fmaf(dx, f, ax);
                    ay = fmaf(dy, f, ay);
                    az = fmaf(dz, f, az);
                }
            }
            double sx = warp_sum((double)ax);
            double sy = warp_sum((double)ay);
            double sz = warp_sum((double)az);
            const size_t gi = (size_t)ustart + ti;
            if (lane == 0) {
                if (flushed_before) {
                    sx += A.facc[3 * gi + 0];
                    sy += A.facc[3 * gi + 1];
                    sz += A.facc[3 * gi + 2];
                }
                if (last) {
                    const float4 L = Lslot[sl];
                    const double m = (double)t.w;
                    A.fx[gi] = (float)(m * ((double)L.y + sx));
                    A.fy[gi] = (float)(m * ((double)L.z + sy));
                    A.fz[gi] = (float)(m * ((double)L.w + sz));
                } else {
                    A.facc[3 * gi + 0] = sx;
                    A.facc[3 * gi + 1] = sy;
                    A.facc[3 * gi + 2] = sz;
                }
            }
        }
    }
    if (!last) flushed_before = true;
    __syncwarp();
}

__global__ void __launch_bounds__(kTravThreads) k_traverse(TravArgs A) {
    __shared__ WarpSmem smem[kTravWarps];
    const uint32_t lane = lane_id();
    const uint32_t lt_mask = lanemask_lt();
    WarpSmem& sm = smem[threadIdx.x >> 5];
    const TreeView& tv = A.tv;
    const int k = A.level;
    const float theta2 = __fmul_rn(A.theta, A.theta);
    const uint32_t gbase = tv.lvl_base[k - 1];
    const uint32_t ngroups = A.status->lvl_count[k - 1];
    if (A.status->err & (PSG_ERR_NODES | PSG_ERR_SORT_SPIN)) return;

    for (;;) {
        uint32_t g0 = 0;
        if (lane == 0) g0 = atomicAdd(&A.status->work[k], (uint32_t)kGroupBatch);
        g0 = __shfl_sync(0xFFFFFFFFu, g0, 0);
        if (g0 >= ngroups) break;
#pragma unroll 1
        for (uint32_t g = g0; g < g0 + kGroupBatch && g < ngroups; ++g) {
            const uint32_t pid = gbase + g;
            const uint4 pinf = tv.info[pid];
            const uint32_t nc = flags_nchild(pinf.w);
            if (nc == 0) continue;
            const uint32_t fc = pinf.z;
            if (lane < nc) {
                sm.cgeo[lane] = tv.geo[fc + lane];
                sm.cinfo[lane] = tv.info[fc + lane];
            }
            __syncwarp();
            // slot masks: which children are targets, which are leaves
            uint32_t leaf_mask = 0, tgt_mask = 0;
            for (uint32_t q = 0; q < nc; ++q) {
                const bool lf = flags_nchild(sm.cinfo[q].w) == 0;
                leaf_mask |= (uint32_t)lf << q;
            }
            tgt_mask = (k == 1) ? leaf_mask : ((1u << nc) - 1u);
            const uint32_t int_mask = tgt_mask & ~leaf_mask;
            if (tgt_mask == 0) continue;
            const float4 Lp = tv.lt[pid];

            // candidate count and near-list reservation for internal children
            const uint32_t* nsl = nullptr;
            uint32_t nsn = 0, cand_total = 1;
            if (k >= 3) {
                nsl = A.ns_in + tv.ns_off[pid];
                nsn = tv.ns_cnt[pid];
                uint32_t c = 0;
                for (uint32_t e = lane; e < nsn; e += 32) {
                    const uint32_t nch = flags_nchild(tv.info[nsl[e]].w);
                    c += nch ? nch : 1u;
                }
                cand_total = warp_sum(c);
            }
            const uint32_t n_int = __popc(int_mask);
            unsigned long long ns_base = 0;
            bool ns_ok = true;
            if (n_int && cand_total) {
                unsigned long long need = (unsigned long long)n_int * cand_total;
                if (lane == 0) ns_base = atomicAdd(&A.status->ns_used[k], need);
                ns_base = __shfl_sync(0xFFFFFFFFu, ns_base, 0);
                if (ns_base + need > A.ns_cap) {
                    ns_ok = false;
                    if (lane == 0) set_err(A.status, PSG_ERR_NS_OVERFLOW);
                }
            }
            uint32_t ns_cnt[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) ns_cnt[q] = 0;
            M2LAcc acc;
#pragma unroll
            for (int q = 0; q < 8; ++q) acc.v[q][0] = acc.v[q][1] = acc.v[q][2] = 0.f;
            uint32_t dbg_m2l[8], dbg_p2p[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) dbg_m2l[q] = dbg_p2p[q] = 0;
            uint32_t ssize = 0, np = 0;
            bool flushed = false;

            // ---------- DFS step over the stack (leaf targets vs internal s) ----------
            auto dfs_step = [&]() {
                int room = ((int)kStackCap - kStackSlack - (int)ssize) / 7;
                uint32_t kp = (uint32_t)min(32, min((int)ssize, max(1, room)));
                uint32_t ent = 0;
                const bool act = lane < kp;
                if (act) ent = sm.stk[ssize - kp + lane];
                ssize -= kp;
                __syncwarp();
                const uint32_t slot = ent >> 28;
                uint4 sinf = make_uint4(0, 0, 0, 0);
                if (act) sinf = tv.info[ent & kNodeMask];
                const uint32_t snch = act ? flags_nchild(sinf.w) : 0u;
                const float4 ug = sm.cgeo[slot];
#pragma unroll 1
                for (uint32_t c = 0; c < 8; ++c) {
                    const bool v = c < snch;
                    if (!__any_sync(0xFFFFFFFFu, v)) break;
                    bool sep = false, p2p = false, push = false;
                    uint32_t sc = 0;
                    if (v) {
                        sc = sinf.z + c;
                        const float4 sg = tv.geo[sc];
                        float dx, dy, dz, d2;
                        sep = mac_separated(ug.x, ug.y, ug.z, ug.w, sg.x, sg.y, sg.z, sg.w,
                                            theta2, dx, dy, dz, d2);
                        if (sep) {
                            float fx, fy, fz;
                            m2l_field(dx, dy, dz, d2, tv.mp[sc], fx, fy, fz);
                            acc_add_dyn(acc, slot, fx, fy, fz);
                        } else if (flags_nchild(tv.info[sc].w) == 0) {
                            p2p = true;
                        } else {
                            push = true;
                        }
                    }
                    if (A.debug) {
#pragma unroll
                        for (int q = 0; q < 8; ++q) {
                            dbg_m2l[q] += __popc(__ballot_sync(0xFFFFFFFFu, sep && slot == (uint32_t)q));
                            dbg_p2p[q] += __popc(__ballot_sync(0xFFFFFFFFu, p2p && slot == (uint32_t)q));
                        }
                    }
                    const uint32_t pm = __ballot_sync(0xFFFFFFFFu, p2p);
                    if (pm) {
                        if (np + __popc(pm) > (uint32_t)kP2PBuf) {
                            p2p_flush(A, sm, np, tgt_mask & leaf_mask, false, flushed, nullptr);
                            np = 0;
                        }
                        if (p2p) sm.p2p[np + __popc(pm & lt_mask)] = (slot << 28) | sc;
                        np += __popc(pm);
                    }
                    const uint32_t qm = __ballot_sync(0xFFFFFFFFu, push);
                    if (qm) {
                        if (ssize + __popc(qm) > (uint32_t)kStackCap) {
                            if (lane == 0) set_err(A.status, PSG_ERR_STACK);
                        } else {
                            if (push) sm.stk[ssize + __popc(qm & lt_mask)] = (slot << 28) | sc;
                            ssize += __popc(qm);
                        }
                    }
                    __syncwarp();
                }
                if (A.debug && lane == 0) atomicMax(&A.status->max_stack, ssize);
            };

            // ---------- phase A: candidates x children ----------
            const uint32_t n_chunks = (k >= 3) ? (nsn + 31) / 32 : 1u;
#pragma unroll 1
            for (uint32_t ch = 0; ch < n_chunks; ++ch) {
                uint32_t tot;
                if (k >= 3) {
                    const uint32_t e = ch * 32 + lane;
                    uint32_t s0 = 0, c = 0, fcs = 0;
                    bool lf = false;
                    if (e < nsn) {
                        s0 = nsl[e];
                        const uint4 si = tv.info[s0];
                        const uint32_t nch = flags_nchild(si.w);
                        lf = nch == 0;
                        c = lf ? 1u : nch;
                        fcs = si.z;
                    }
                    const uint32_t inc = warp_incl_scan(c);
                    tot = __shfl_sync(0xFFFFFFFFu, inc, 31);
                    const uint32_t ex = inc - c;
                    if (lf) sm.cand[ex] = s0;
                    else for (uint32_t q = 0; q < c; ++q) sm.cand[ex + q] = fcs + q;
                } else {
                    tot = 1;
                    if (lane == 0) sm.cand[0] = 0;  // the root
                }
                __syncwarp();
#pragma unroll 1
                for (uint32_t j0 = 0; j0 < tot; j0 += 32) {
                    const uint32_t j = j0 + lane;
                    const bool valid = j < tot;
                    uint32_t s = 0;
                    float4 sg = make_float4(0.f, 0.f, 0.f, 0.f), smp = sg;
                    bool sleaf = false;
                    if (valid) {
                        s = sm.cand[j];
                        sg = tv.geo[s];
                        smp = tv.mp[s];
                        sleaf = flags_nchild(tv.info[s].w) == 0;
                    }
#pragma unroll
                    for (uint32_t q = 0; q < 8; ++q) {
                        if (!((tgt_mask >> q) & 1u)) continue;
                        const float4 ug = sm.cgeo[q];
                        float dx, dy, dz, d2;
                        const bool sep = valid && mac_separated(ug.x, ug.y, ug.z, ug.w, sg.x, sg.y,
                                                                sg.z, sg.w, theta2, dx, dy, dz, d2);
                        if (sep) {
                            float fx, fy, fz;
                            m2l_field(dx, dy, dz, d2, smp, fx, fy, fz);
                            acc.v[q][0] += fx;
                            acc.v[q][1] += fy;
                            acc.v[q][2] += fz;
                        }
                        const bool near = valid && !sep;
                        if (A.debug) dbg_m2l[q] += __popc(__ballot_sync(0xFFFFFFFFu, sep));
                        if ((int_mask >> q) & 1u) {
                            const uint32_t nm = __ballot_sync(0xFFFFFFFFu, near);
                            if (nm && ns_ok) {
                                const uint32_t sub = __popc(int_mask & ((1u << q) - 1u));
                                const unsigned long long off =
                                    ns_base + (unsigned long long)sub * cand_total + ns_cnt[q];
                                if (near) A.ns_out[off + __popc(nm & lt_mask)] = s;
                            }
                            ns_cnt[q] += __popc(nm);
                        } else {
                            const bool p2p = near && sleaf;
                            const bool push = near && !sleaf;
                            const uint32_t pm = __ballot_sync(0xFFFFFFFFu, p2p);
                            if (A.debug) dbg_p2p[q] += __popc(pm);
                            if (pm) {
                                if (np + __popc(pm) > (uint32_t)kP2PBuf) {
                                    p2p_flush(A, sm, np, tgt_mask & leaf_mask, false, flushed,
                                              nullptr);
                                    np = 0;
                                }
                                if (p2p) sm.p2p[np + __popc(pm & lt_mask)] = (q << 28) | s;
                                np += __popc(pm);
                            }
                            const uint32_t qm = __ballot_sync(0xFFFFFFFFu, push);
                            if (qm) {
                                if (ssize + __popc(qm) > (uint32_t)kStackCap) {
                                    if (lane == 0) set_err(A.status, PSG_ERR_STACK);
                                } else {
                                    if (push) sm.stk[ssize + __popc(qm & lt_mask)] = (q << 28) | s;
                                    ssize += __popc(qm);
                                }
                            }
                        }
                        __syncwarp();
                    }
                    // leave room for the next sub-chunk's pushes (<= 8 slots x 32)
                    while (ssize > (uint32_t)(kStackCap - kStackSlack - 8 * 32)) dfs_step();
                }
                __syncwarp();
            }
            // ---------- phase B: finish the leaf-target recursions ----------
            while (ssize > 0) dfs_step();

            // ---------- L2L / outputs ----------
            __shared__ float4 s_L[kTravWarps][8];
#pragma unroll
            for (uint32_t q = 0; q < 8; ++q) {
                if (!((tgt_mask >> q) & 1u)) continue;
                const float ax = warp_sum(acc.v[q][0]);
                const float ay = warp_sum(acc.v[q][1]);
                const float az = warp_sum(acc.v[q][2]);
                // L(u) = M2L(u) + L(parent)  (polesitter.h:1248-1250)
                const float4 L = make_float4(0.f, __fadd_rn(ax, Lp.y), __fadd_rn(ay, Lp.z),
                                             __fadd_rn(az, Lp.w));
                if (lane == 0) {
                    const uint32_t u = fc + q;
                    tv.lt[u] = L;
                    s_L[threadIdx.x >> 5][q] = L;
                    if ((int_mask >> q) & 1u) {
                        const uint32_t sub = __popc(int_mask & ((1u << q) - 1u));
                        tv.ns_off[u] = (uint32_t)(ns_base + (unsigned long long)sub * cand_total);
                        tv.ns_cnt[u] = ns_ok ? ns_cnt[q] : 0u;
                    }
                    if (A.debug) {
                        tv.dbg_m2l[u] = dbg_m2l[q];
                        tv.dbg_p2p[u] = dbg_p2p[q];
                    }
                }
            }
            __syncwarp();
            if (tgt_mask & leaf_mask) {
                p2p_flush(A, sm, np, tgt_mask & leaf_mask, true, flushed, s_L[threadIdx.x >> 5]);
                np = 0;
            }
            if (A.debug && lane == 0) {
                unsigned long long m = 0, p = 0;
                for (int q = 0; q < 8; ++q) {
                    m += dbg_m2l[q];
                    p += dbg_p2p[q];
                }
                atomicAdd(&A.status->stat[PSG_STAT_M2L], m);
                atomicAdd(&A.status->stat[PSG_STAT_P2P_PAIRS], p);
            }
            __syncwarp();
        }
    }
}

void launch_traverse_level(const TravLaunch& L, int level, const uint32_t* ns_in, uint32_t* ns_out,
                           int grid, cudaStream_t st) {
    TravArgs A;
    A.tv = L.tv;
    A.xyzm = L.xyzm;
    A.fx = L.fx;
    A.fy = L.fy;
    A.fz = L.fz;
    A.ns_in = ns_in;
    A.ns_out = ns_out;
    A.ns_cap = L.ns_cap;
    A.facc = L.facc;
    A.status = L.status;
    A.theta = L.theta;
    A.level = level;
    A.debug = L.debug;
    k_traverse<<<grid, kTravThreads, 0, st>>>(A);
}

int traverse_threads() { return kTravThreads; }
const void* traverse_kernel_ptr() { return (const void*)k_traverse; }

}  // namespace psg
