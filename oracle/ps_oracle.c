/*
 * ORACLE (test infrastructure, not product): a CPU restatement of the
 * polesitter FMM tick, ps_prepare_particles + ps_calc_forces, as the
 * reference computes it when built with PS_MULTITHREADING (the build every
 * reference test and benchmark uses, tests/main.c:7-9).
 *
 * Only tests/, the smoke check and bench.py's CPU baseline load this code,
 * and only as a checker.  It is compiled with strict IEEE arithmetic (no
 * fast-math, no FMA contraction) by oracle/build_oracle.sh and is pinned
 * against the reference itself (oracle/_ref, built from the reference's own
 * header) by tests/test_oracle.py: Morton codes, order, ids, tree, per-node
 * fields and forces agree bit-for-bit with the strict build of the reference
 * and within 2e-7 relative L2 with its fast-math build.
 *
 * Beyond the reference's outputs it records what the GPU kernels must agree
 * on exactly: per-node M2L pair counts, the P2P leaf-pair list and the
 * traversal totals (MAC tests, M2L pairs, P2P pairs and particle pairs).
 *
 * Every function cites the reference lines it restates (src/polesitter.h).
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#if defined(__AVX2__)
#include <immintrin.h>
#endif

#define PSO_API __attribute__((visibility("default")))
#define PSO_MAX_DEPTH 10 /* polesitter.h:882-883 */

/* ---------------------------------------------------------------------
 * Morton code: 10-bit expand (polesitter.h:778-787) and interleave with x on
 * bit 0, y on bit 1, z on bit 2 (:792-799).
 * ------------------------------------------------------------------- */
static uint32_t pso_expand10(uint32_t v) {
    v &= 0x3FFu;
    v = (v | (v << 16)) & 0x030000FFu;
    v = (v | (v << 8)) & 0x0300F00Fu;
    v = (v | (v << 4)) & 0x030C30C3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

PSO_API uint32_t pso_morton_encode(uint32_t x, uint32_t y, uint32_t z) {
    return pso_expand10(x) | (pso_expand10(y) << 1) | (pso_expand10(z) << 2);
}

/* round-to-nearest-even float -> int, as _mm256_cvtps_epi32 under the default
 * MXCSR mode (polesitter.h:2056-2058) */
static int32_t pso_cvt_rne(float v) { return (int32_t)nearbyintf(v); }

/* quantisation variants of polesitter.h:2013-2157 */
enum { PSO_MORTON_AVX2 = 0, PSO_MORTON_NEON = 1, PSO_MORTON_SCALAR = 2 };

static uint32_t pso_q_vec(float v, float min_b, float scale, int trunc) {
    /* (v - min) * (1023 / range), clamped with max(0, min(., 1023)) and
     * converted: AVX2 rounds to nearest even (:2046-2058), NEON truncates
     * (:2101-2113). */
    float q = (v - min_b) * scale;
    q       = (q < 1023.0F) ? q : 1023.0F;
    q       = (0.0F > q) ? 0.0F : q;
    return (uint32_t)(trunc ? (int32_t)q : pso_cvt_rne(q));
}

static uint32_t pso_q_scalar(float v, float min_b, float range) {
    /* (int)(((v - min) / range) * 1023), then clamp to [0, 1023]
     * (:2133-2153) */
    int q = (int)(((v - min_b) / range) * 1023.0F);
    if (q < 0) {
        q = 0;
    }
    if (q > 1023) {
        q = 1023;
    }
    return (uint32_t)q;
}

/* ps_prepare_particles (polesitter.h:1911-2170).  The bounding box is the
 * min / max over x, y and z jointly (:1918-2006), the range is clamped to at
 * least 1e-3 (:2008-2011).  The vector path covers whole groups of `lanes`
 * particles (8 for AVX2, 4 for NEON), the scalar formula covers the
 * remainder (:2132-2157); the scalar build uses the scalar formula
 * throughout. */
PSO_API int pso_prepare(size_t n, const float* x, const float* y,
                        const float* z, uint32_t* codes, float* out_min,
                        float* out_max, float* out_range, int variant) {
    if (n == 0 || !codes) {
        return -2; /* PS_EINVAL, :1914 */
    }
    float mn = FLT_MAX;
    float mx = -FLT_MAX;
    for (size_t i = 0; i < n; ++i) {
        const float v[3] = {x[i], y[i], z[i]};
        for (int a = 0; a < 3; ++a) {
            if (v[a] < mn) {
                mn = v[a];
            }
            if (v[a] > mx) {
                mx = v[a];
            }
        }
    }
    float range = mx - mn;
    if (range < 0.001F) {
        range = 0.001F;
    }
    size_t lanes = (variant == PSO_MORTON_AVX2)   ? 8
                   : (variant == PSO_MORTON_NEON) ? 4
                                                  : 0;
    size_t vec_end = lanes ? (n / lanes) * lanes : 0;
    float  scale   = 1023.0F / range;
    int    trunc   = (variant == PSO_MORTON_NEON);
    for (size_t i = 0; i < n; ++i) {
        uint32_t qx, qy, qz;
        if (i < vec_end) {
            qx = pso_q_vec(x[i], mn, scale, trunc);
            qy = pso_q_vec(y[i], mn, scale, trunc);
            qz = pso_q_vec(z[i], mn, scale, trunc);
        } else {
            qx = pso_q_scalar(x[i], mn, range);
            qy = pso_q_scalar(y[i], mn, range);
            qz = pso_q_scalar(z[i], mn, range);
        }
        codes[i] = pso_morton_encode(qx, qy, qz);
    }
    if (out_min) {
        *out_min = mn;
    }
    if (out_max) {
        *out_max = mx;
    }
    if (out_range) {
        *out_range = range;
    }
    return 0;
}

/* ---------------------------------------------------------------------
 * Stable ascending sort by the full 32-bit code; co-permutes
 * codes, id, x, y, z, mass (polesitter.h:1588-1693, four stable 8-bit LSD
 * passes; any stable sort gives the same permutation).
 * ------------------------------------------------------------------- */
PSO_API void pso_sort(size_t n, uint32_t* codes, uint32_t* id, float* x,
                      float* y, float* z, float* m) {
    uint32_t* perm = (uint32_t*)malloc(n * sizeof(uint32_t));
    uint32_t* tmp  = (uint32_t*)malloc(n * sizeof(uint32_t));
    uint32_t* key  = (uint32_t*)malloc(n * sizeof(uint32_t));
    uint32_t* ktmp = (uint32_t*)malloc(n * sizeof(uint32_t));
    for (size_t i = 0; i < n; ++i) {
        perm[i] = (uint32_t)i;
        key[i]  = codes[i];
    }
    for (int pass = 0; pass < 4; ++pass) {
        size_t cnt[257] = {0};
        int    sh       = pass * 8;
        for (size_t i = 0; i < n; ++i) {
            cnt[((key[i] >> sh) & 0xFFu) + 1]++;
        }
        for (int b = 0; b < 256; ++b) {
            cnt[b + 1] += cnt[b];
        }
        for (size_t i = 0; i < n; ++i) {
            size_t dst = cnt[(key[i] >> sh) & 0xFFu]++;
            ktmp[dst]  = key[i];
            tmp[dst]   = perm[i];
        }
        uint32_t* t = key;
        key         = ktmp;
        ktmp        = t;
        t           = perm;
        perm        = tmp;
        tmp         = t;
    }
    float*    fb = (float*)malloc(n * sizeof(float));
    uint32_t* ub = (uint32_t*)malloc(n * sizeof(uint32_t));
#define PSO_PERMUTE(arr, buf)                                                  \
    do {                                                                       \
        for (size_t i = 0; i < n; ++i) {                                       \
            (buf)[i] = (arr)[perm[i]];                                         \
        }                                                                      \
        memcpy((arr), (buf), n * sizeof((arr)[0]));                            \
    } while (0)
    PSO_PERMUTE(codes, ub);
    PSO_PERMUTE(id, ub);
    PSO_PERMUTE(x, fb);
    PSO_PERMUTE(y, fb);
    PSO_PERMUTE(z, fb);
    PSO_PERMUTE(m, fb);
#undef PSO_PERMUTE
    free(fb);
    free(ub);
    free(perm);
    free(tmp);
    free(key);
    free(ktmp);
}

/* ---------------------------------------------------------------------
 * Tree: level-major, each level in Morton order.
 * ------------------------------------------------------------------- */
typedef struct {
    float    x, y, z, hw;        /* ps_node_t x,y,z,half_width (:362-368) */
    float    mp[4];              /* multipole (:370) */
    float    l_m2l[4];           /* M2L sum received by this node */
    float    l_tot[4];           /* local_exp after the downward pass */
    float    g_m2l[6], g_tot[6]; /* closure order 1: field gradient (xx yy zz xy xz yz) */
    uint32_t start, count;       /* particle range */
    uint32_t first_child, nchild;
    uint32_t parent;
    int32_t  depth, octant;
    uint32_t m2l_cnt;            /* M2L pairs with this node as target */
    uint32_t p2p_cnt;            /* P2P leaf pairs with this node as target */
} pso_node_t;

typedef struct {
    pso_node_t* nodes;
    size_t      n_nodes, cap;
    uint32_t    level_start[PSO_MAX_DEPTH + 2];
    /* P2P leaf pairs in the reference's evaluation order */
    uint32_t*   p2p_t;
    uint32_t*   p2p_s;
    size_t      n_p2p, p2p_cap;
    /* traversal totals */
    uint64_t    mac_tests, m2l_pairs, p2p_interactions;
    /* sorted particle view used by the passes */
    const float *x, *y, *z, *m;
    float        theta;
    int          accum_mode; /* 0: reference lane structure; 1: plain */
    int          order;      /* closure: 0 reference (order-0 local), 1 order-1 */
    uint32_t     leaf_cap;   /* split nodes holding more than this (0 or 1: the reference) */
    float*       feat;       /* closure: raw per-particle features, 16 each */
} pso_ctx_t;

PSO_API void* pso_new(void) { return calloc(1, sizeof(pso_ctx_t)); }

PSO_API void pso_free(void* h) {
    pso_ctx_t* c = (pso_ctx_t*)h;
    if (!c) {
        return;
    }
    free(c->nodes);
    free(c->p2p_t);
    free(c->p2p_s);
    free(c);
}

static uint32_t pso_push_node(pso_ctx_t* c) {
    if (c->n_nodes == c->cap) {
        c->cap   = c->cap ? 2 * c->cap : 1024;
        c->nodes = (pso_node_t*)realloc(c->nodes, c->cap * sizeof(pso_node_t));
    }
    memset(&c->nodes[c->n_nodes], 0, sizeof(pso_node_t));
    return (uint32_t)c->n_nodes++;
}

/* first index in [lo, hi) whose octal digit at `shift` is >= target
 * (ps_impl_find_split, polesitter.h:886-903) */
static size_t pso_find_split(const uint32_t* codes, size_t lo, size_t hi,
                             int shift, uint32_t target) {
    while (lo < hi) {
        size_t mid = lo + ((hi - lo) / 2);
        if (((codes[mid] >> shift) & 7u) < target) {
            lo = mid + 1;
        } else {
            hi = mid;
        }
    }
    return lo;
}

/* ps_impl_build_tree (polesitter.h:906-967) done breadth-first: a node at
 * depth d is a leaf iff d == 10 or it holds <= 1 particle (:911-916) --
 * <= leaf_cap particles with pso_set_leaf_cap, an extension that still
 * splits a root holding two or more;
 * otherwise one child per non-empty octant of digit (code >> (27-3d)) & 7,
 * in octant order, centred at parent +/- hw/2 per axis bit (x = bit 0,
 * y = bit 1, z = bit 2) with hw_child = hw * 0.5 (:935-939). */
static void pso_build(pso_ctx_t* c, const uint32_t* codes, size_t n, float cx,
                      float cy, float cz, float hw) {
    c->n_nodes    = 0;
    uint32_t root = pso_push_node(c);
    pso_node_t* r = &c->nodes[root];
    r->x = cx;
    r->y = cy;
    r->z = cz;
    r->hw = hw;
    r->start = 0;
    r->count = (uint32_t)n;
    r->parent = 0xFFFFFFFFu;
    r->octant = -1;
    c->level_start[0] = 0;
    const uint32_t cap = c->leaf_cap > 1 ? c->leaf_cap : 1u;
    size_t lvl_lo = 0, lvl_hi = 1;
    for (int d = 0; d <= PSO_MAX_DEPTH; ++d) {
        c->level_start[d + 1] = (uint32_t)lvl_hi;
        for (size_t k = lvl_lo; k < lvl_hi; ++k) {
            pso_node_t p = c->nodes[k];
            if (d == PSO_MAX_DEPTH || p.count <= (d == 0 ? 1u : cap)) {
                c->nodes[k].nchild      = 0;
                c->nodes[k].first_child = 0;
                continue;
            }
            int    shift = 27 - (3 * d);
            size_t cur   = p.start;
            size_t end   = (size_t)p.start + p.count;
            c->nodes[k].first_child = (uint32_t)c->n_nodes;
            for (uint32_t oct = 0; oct < 8; ++oct) {
                size_t oe = pso_find_split(codes, cur, end, shift, oct + 1);
                if (oe > cur) {
                    uint32_t    ci = pso_push_node(c);
                    pso_node_t* ch = &c->nodes[ci];
                    pso_node_t* pp = &c->nodes[k];
                    float       h  = pp->hw * 0.5F;
                    ch->x      = pp->x + ((oct & 1) ? h : -h);
                    ch->y      = pp->y + ((oct & 2) ? h : -h);
                    ch->z      = pp->z + ((oct & 4) ? h : -h);
                    ch->hw     = h;
                    ch->start  = (uint32_t)cur;
                    ch->count  = (uint32_t)(oe - cur);
                    ch->parent = (uint32_t)k;
                    ch->depth  = d + 1;
                    ch->octant = (int32_t)oct;
                    pp->nchild++;
                }
                cur = oe;
                if (cur == end) {
                    break;
                }
            }
        }
        lvl_lo = lvl_hi;
        lvl_hi = c->n_nodes;
        if (lvl_lo == lvl_hi) {
            for (int e = d + 2; e <= PSO_MAX_DEPTH + 1; ++e) {
                c->level_start[e] = (uint32_t)lvl_hi;
            }
            break;
        }
    }
}

static int pso_is_leaf(const pso_node_t* n) { return n->nchild == 0; }

/* ps_impl_fmm_upward_pass (polesitter.h:971-1046): P2M sums
 * m0 = sum m, m_k = sum m * (x_k - c_k) over the leaf's particles in order;
 * M2M adds children in octant order, P_k += C_k + C0 * (c_child - c_parent)_k.
 * Bottom-up over levels gives the same per-node operation order. */
static void pso_upward(pso_ctx_t* c) {
    for (size_t kk = c->n_nodes; kk-- > 0;) {
        pso_node_t* nd = &c->nodes[kk];
        if (pso_is_leaf(nd)) {
            float m0 = 0.0F, mx = 0.0F, my = 0.0F, mz = 0.0F;
            for (uint32_t i = 0; i < nd->count; ++i) {
                uint32_t idx  = nd->start + i;
                float    mass = c->m[idx];
                float    dx   = c->x[idx] - nd->x;
                float    dy   = c->y[idx] - nd->y;
                float    dz   = c->z[idx] - nd->z;
                m0 += mass;
                mx += mass * dx;
                my += mass * dy;
                mz += mass * dz;
            }
            nd->mp[0] = m0;
            nd->mp[1] = mx;
            nd->mp[2] = my;
            nd->mp[3] = mz;
        } else {
            float p0 = 0.0F, px = 0.0F, py = 0.0F, pz = 0.0F;
            for (uint32_t j = 0; j < nd->nchild; ++j) {
                const pso_node_t* ch = &c->nodes[nd->first_child + j];
                float dx = ch->x - nd->x;
                float dy = ch->y - nd->y;
                float dz = ch->z - nd->z;
                p0 += ch->mp[0];
                px += ch->mp[1] + (ch->mp[0] * dx);
                py += ch->mp[2] + (ch->mp[0] * dy);
                pz += ch->mp[3] + (ch->mp[0] * dz);
            }
            nd->mp[0] = p0;
            nd->mp[1] = px;
            nd->mp[2] = py;
            nd->mp[3] = pz;
        }
    }
}

/* multipole acceptance criterion (polesitter.h:1056-1064, :1265-1273):
 * separated iff ((dx*dx + dy*dy) + dz*dz) > (theta*theta) * (hw_sum*hw_sum),
 * every operation rounded to nearest, strict '>'. */
static int pso_mac(const pso_node_t* t, const pso_node_t* s, float theta,
                   float* dx, float* dy, float* dz, float* d2) {
    *dx = s->x - t->x;
    *dy = s->y - t->y;
    *dz = s->z - t->z;
    *d2 = ((*dx * *dx) + (*dy * *dy)) + (*dz * *dz);
    float hs = t->hw + s->hw;
    return *d2 > ((theta * theta) * (hs * hs));
}

static void pso_push_p2p(pso_ctx_t* c, uint32_t t, uint32_t s) {
    if (c->n_p2p == c->p2p_cap) {
        c->p2p_cap = c->p2p_cap ? 2 * c->p2p_cap : 4096;
        c->p2p_t   = (uint32_t*)realloc(c->p2p_t, c->p2p_cap * sizeof(uint32_t));
        c->p2p_s   = (uint32_t*)realloc(c->p2p_s, c->p2p_cap * sizeof(uint32_t));
    }
    c->p2p_t[c->n_p2p] = t;
    c->p2p_s[c->n_p2p] = s;
    c->n_p2p++;
}

/* ps_impl_fmm_interaction_pass (polesitter.h:1050-1146).  The P2P pass
 * (:1258-1494) walks the same pairs with the same MAC, so one walk records
 * both: M2L is applied on the spot (same order as the reference), leaf x leaf
 * non-separated pairs are queued for P2P in the order the P2P pass visits
 * them. */
static void pso_interact(pso_ctx_t* c, uint32_t ti, uint32_t si) {
    pso_node_t*       t = &c->nodes[ti];
    const pso_node_t* s = &c->nodes[si];
    float             dx, dy, dz, d2;
    c->mac_tests++;
    if (pso_mac(t, s, c->theta, &dx, &dy, &dz, &d2)) {
        /* M2L, :1065-1092 */
        float soft   = d2 + 0.1F;
        float dist   = sqrtf(soft);
        float inv_r3 = 1.0F / (dist * soft);
        float inv_r5 = inv_r3 / soft;
        float m0 = s->mp[0], mx = s->mp[1], my = s->mp[2], mz = s->mp[3];
        float fmx   = m0 * dx * inv_r3;
        float fmy   = m0 * dy * inv_r3;
        float fmz   = m0 * dz * inv_r3;
        float mdr   = (mx * dx) + (my * dy) + (mz * dz);
        float coeff = 3.0F * mdr * inv_r5;
        float fdx   = (mx * inv_r3) - (dx * coeff);
        float fdy   = (my * inv_r3) - (dy * coeff);
        float fdz   = (mz * inv_r3) - (dz * coeff);
        if (c->order >= 1) {
            /* closure order 1: gradient of the monopole field at the target
             * centre, d(m0 d ir3)/d(target) = m0 (3 d d^T ir5 - I ir3) */
            float g3 = 3.0F * m0 * inv_r5;
            float gi = m0 * inv_r3;
            t->g_m2l[0] += g3 * dx * dx - gi;
            t->g_m2l[1] += g3 * dy * dy - gi;
            t->g_m2l[2] += g3 * dz * dz - gi;
            t->g_m2l[3] += g3 * dx * dy;
            t->g_m2l[4] += g3 * dx * dz;
            t->g_m2l[5] += g3 * dy * dz;
        }
        t->l_m2l[1] += fmx + fdx;
        t->l_m2l[2] += fmy + fdy;
        t->l_m2l[3] += fmz + fdz;
        t->m2l_cnt++;
        c->m2l_pairs++;
        return;
    }
    int tl = pso_is_leaf(t);
    int sl = pso_is_leaf(s);
    if (tl && sl) {
        t->p2p_cnt++;
        pso_push_p2p(c, ti, si);
        return;
    }
    if (tl) {
        for (uint32_t j = 0; j < s->nchild; ++j) {
            pso_interact(c, ti, s->first_child + j);
        }
    } else if (sl) {
        for (uint32_t j = 0; j < t->nchild; ++j) {
            pso_interact(c, t->first_child + j, si);
        }
    } else {
        uint32_t tf = t->first_child, tn = t->nchild;
        uint32_t sf = s->first_child, sn = s->nchild;
        for (uint32_t i = 0; i < tn; ++i) {
            for (uint32_t j = 0; j < sn; ++j) {
                pso_interact(c, tf + i, sf + j);
            }
        }
    }
}

/* ps_impl_dispatch_fmm (polesitter.h:1772-1801, called with target depth 2
 * from :1883-1885): every node at depth 2, and every leaf above it, is paired
 * with the root; the single-threaded build (:1888) pairs (root, root)
 * instead. */
static void pso_dispatch(pso_ctx_t* c, uint32_t ti, int depth, int mt) {
    const pso_node_t* t = &c->nodes[ti];
    if (!mt || depth == 2 || pso_is_leaf(t)) {
        pso_interact(c, ti, 0);
        return;
    }
    for (uint32_t j = 0; j < t->nchild; ++j) {
        pso_dispatch(c, t->first_child + j, depth + 1, mt);
    }
}

/* leaf x leaf direct sum (polesitter.h:1279-1449).  For each target
 * particle the source leaf is walked in chunks of 8 with the AVX2 lane
 * arithmetic (:1299-1356: rsqrt estimate, (dx^2+dy^2)+(dz^2+eps), per-lane
 * sums reduced in lane order) and the remainder with the scalar formula
 * (:1424-1444: ((dx^2+dy^2)+dz^2)+eps, 1/sqrtf).  accum_mode 1 uses the
 * scalar formula for every source particle. */
static void pso_p2p_leaves(pso_ctx_t* c, const pso_node_t* t,
                         const pso_node_t* s, float* fx, float* fy,
                         float* fz) {
    for (uint32_t i = 0; i < t->count; ++i) {
        uint32_t ti = t->start + i;
        float    tx = c->x[ti], ty = c->y[ti], tz = c->z[ti], tm = c->m[ti];
        float    f_x = 0.0F, f_y = 0.0F, f_z = 0.0F;
        uint32_t j   = 0;
#if defined(__AVX2__)
        if (c->accum_mode == 0) {
            __m256 vtx = _mm256_set1_ps(tx), vty = _mm256_set1_ps(ty);
            __m256 vtz = _mm256_set1_ps(tz), eps = _mm256_set1_ps(0.1F);
            __m256 ax = _mm256_setzero_ps(), ay = _mm256_setzero_ps();
            __m256 az = _mm256_setzero_ps();
            for (; j + 7 < s->count; j += 8) {
                uint32_t si = s->start + j;
                __m256   px = _mm256_sub_ps(_mm256_loadu_ps(&c->x[si]), vtx);
                __m256   py = _mm256_sub_ps(_mm256_loadu_ps(&c->y[si]), vty);
                __m256   pz = _mm256_sub_ps(_mm256_loadu_ps(&c->z[si]), vtz);
                __m256   r2 = _mm256_add_ps(
                    _mm256_add_ps(_mm256_mul_ps(px, px), _mm256_mul_ps(py, py)),
                    _mm256_add_ps(_mm256_mul_ps(pz, pz), eps));
                __m256 ir  = _mm256_rsqrt_ps(r2);
                __m256 ir3 = _mm256_mul_ps(_mm256_mul_ps(ir, ir), ir);
                __m256 fm  = _mm256_mul_ps(_mm256_loadu_ps(&c->m[si]), ir3);
                ax = _mm256_add_ps(ax, _mm256_mul_ps(px, fm));
                ay = _mm256_add_ps(ay, _mm256_mul_ps(py, fm));
                az = _mm256_add_ps(az, _mm256_mul_ps(pz, fm));
            }
            float lx[8], ly[8], lz[8];
            _mm256_storeu_ps(lx, ax);
            _mm256_storeu_ps(ly, ay);
            _mm256_storeu_ps(lz, az);
            for (int l = 0; l < 8; ++l) {
                f_x += lx[l];
                f_y += ly[l];
                f_z += lz[l];
            }
        }
#endif
        for (; j < s->count; ++j) {
            uint32_t si   = s->start + j;
            float    p_dx = c->x[si] - tx;
            float    p_dy = c->y[si] - ty;
            float    p_dz = c->z[si] - tz;
            float    r2   = (p_dx * p_dx) + (p_dy * p_dy) + (p_dz * p_dz) + 0.1F;
            float    ir   = 1.0F / sqrtf(r2);
            float    ir3  = ir * ir * ir;
            float    f    = c->m[si] * ir3;
            f_x += p_dx * f;
            f_y += p_dy * f;
            f_z += p_dz * f;
        }
        fx[ti] += tm * f_x;
        fy[ti] += tm * f_y;
        fz[ti] += tm * f_z;
    }
}

/* Closure order 1 (no counterpart in the reference): the downward pass with
 * an order-1 local expansion.  L2L shifts the parent's field to the child's
 * centre, L(u) = M2L(u) + L(p) + G(p) (c_u - c_p), G(u) = M2L_G(u) + G(p);
 * L2P evaluates F_i = m_i (L + G (x_i - c)) at the particle.  With c->feat
 * set it also records each particle's raw closure features: L (3), G (6),
 * x_i - c (3), leaf half width, leaf depth, m_i, 0. */
static void pso_downward_order1(pso_ctx_t* c, size_t n, float* fx, float* fy,
                                float* fz) {
    (void)n;
    for (size_t k = 0; k < c->n_nodes; ++k) {
        pso_node_t* nd = &c->nodes[k];
        for (int a = 0; a < 4; ++a) {
            nd->l_tot[a] = nd->l_m2l[a];
        }
        for (int a = 0; a < 6; ++a) {
            nd->g_tot[a] = nd->g_m2l[a];
        }
        if (k > 0) {
            const pso_node_t* p = &c->nodes[nd->parent];
            const float*      G = p->g_tot;
            float ux = nd->x - p->x, uy = nd->y - p->y, uz = nd->z - p->z;
            nd->l_tot[1] += p->l_tot[1] + (G[0] * ux + G[3] * uy + G[4] * uz);
            nd->l_tot[2] += p->l_tot[2] + (G[3] * ux + G[1] * uy + G[5] * uz);
            nd->l_tot[3] += p->l_tot[3] + (G[4] * ux + G[5] * uy + G[2] * uz);
            for (int a = 0; a < 6; ++a) {
                nd->g_tot[a] += G[a];
            }
        }
        if (!pso_is_leaf(nd)) {
            continue;
        }
        const float* G = nd->g_tot;
        for (uint32_t i = 0; i < nd->count; ++i) {
            uint32_t idx = nd->start + i;
            float ux = c->x[idx] - nd->x, uy = c->y[idx] - nd->y, uz = c->z[idx] - nd->z;
            float lx = nd->l_tot[1] + (G[0] * ux + G[3] * uy + G[4] * uz);
            float ly = nd->l_tot[2] + (G[3] * ux + G[1] * uy + G[5] * uz);
            float lz = nd->l_tot[3] + (G[4] * ux + G[5] * uy + G[2] * uz);
            fx[idx] += c->m[idx] * lx;
            fy[idx] += c->m[idx] * ly;
            fz[idx] += c->m[idx] * lz;
            if (c->feat) {
                float* f = c->feat + 16 * (size_t)idx;
                f[0] = nd->l_tot[1];
                f[1] = nd->l_tot[2];
                f[2] = nd->l_tot[3];
                for (int a = 0; a < 6; ++a) {
                    f[3 + a] = G[a];
                }
                f[9]  = ux;
                f[10] = uy;
                f[11] = uz;
                f[12] = nd->hw;
                f[13] = (float)nd->depth;
                f[14] = c->m[idx];
                f[15] = 0.0F;
            }
        }
    }
}

/* closure mode of the next pso_calc: order 0 = the reference, 1 = order-1
 * local expansion; feat (16 floats per particle) may be NULL */
PSO_API void pso_set_closure(void* h, int order, float* feat) {
    pso_ctx_t* c = (pso_ctx_t*)h;
    c->order = order;
    c->feat  = feat;
}

/* leaf capacity of the next pso_calc's tree: nodes with more than `cap`
 * particles are split (the reference: 1) */
PSO_API void pso_set_leaf_cap(void* h, uint32_t cap) {
    pso_ctx_t* c = (pso_ctx_t*)h;
    c->leaf_cap = cap;
}

/* ps_calc_forces (polesitter.h:1840-1909) on arrays already sorted by
 * pso_sort: build -> upward -> M2L (MT dispatch unless mt == 0) ->
 * downward L2L (:1238-1251, :1820-1835) + L2P (:1224-1233) -> P2P. */
PSO_API int pso_calc(void* h, size_t n, const uint32_t* codes, const float* x,
                     const float* y, const float* z, const float* m, float* fx,
                     float* fy, float* fz, float cx, float cy, float cz,
                     float hw, float theta, int mt, int accum_mode) {
    pso_ctx_t* c = (pso_ctx_t*)h;
    if (!c) {
        return -2;
    }
    c->x = x;
    c->y = y;
    c->z = z;
    c->m = m;
    c->theta      = (theta > 0.0F) ? theta : 1.0F; /* :1707 */
    c->accum_mode = accum_mode;
    c->n_p2p      = 0;
    c->mac_tests = c->m2l_pairs = c->p2p_interactions = 0;
    for (size_t i = 0; i < n; ++i) {
        fx[i] = 0.0F;
        fy[i] = 0.0F;
        fz[i] = 0.0F;
    }
    pso_build(c, codes, n, cx, cy, cz, hw);
    pso_upward(c);
    pso_dispatch(c, 0, 0, mt);
    /* downward: L_total(child) = L_m2l(child) + L_total(parent) */
    if (c->order >= 1) {
        pso_downward_order1(c, n, fx, fy, fz);
    }
    for (size_t k = 0; c->order == 0 && k < c->n_nodes; ++k) {
        pso_node_t* nd = &c->nodes[k];
        for (int a = 0; a < 4; ++a) {
            nd->l_tot[a] = nd->l_m2l[a];
        }
        if (k > 0) {
            const pso_node_t* p = &c->nodes[nd->parent];
            nd->l_tot[1] += p->l_tot[1];
            nd->l_tot[2] += p->l_tot[2];
            nd->l_tot[3] += p->l_tot[3];
        }
        if (pso_is_leaf(nd)) {
            for (uint32_t i = 0; i < nd->count; ++i) {
                uint32_t idx = nd->start + i;
                fx[idx] += m[idx] * nd->l_tot[1];
                fy[idx] += m[idx] * nd->l_tot[2];
                fz[idx] += m[idx] * nd->l_tot[3];
            }
        }
    }
    for (size_t k = 0; k < c->n_p2p; ++k) {
        const pso_node_t* t = &c->nodes[c->p2p_t[k]];
        const pso_node_t* s = &c->nodes[c->p2p_s[k]];
        c->p2p_interactions += (uint64_t)t->count * s->count;
        pso_p2p_leaves(c, t, s, fx, fy, fz);
    }
    return 0;
}

/* ---- accessors ------------------------------------------------------- */

PSO_API size_t pso_num_nodes(void* h) { return ((pso_ctx_t*)h)->n_nodes; }
PSO_API size_t pso_num_p2p(void* h) { return ((pso_ctx_t*)h)->n_p2p; }

PSO_API void pso_stats(void* h, uint64_t* out4) {
    pso_ctx_t* c = (pso_ctx_t*)h;
    out4[0]      = c->mac_tests;
    out4[1]      = c->m2l_pairs;
    out4[2]      = c->n_p2p;
    out4[3]      = c->p2p_interactions;
}

PSO_API void pso_level_starts(void* h, uint32_t* out12) {
    memcpy(out12, ((pso_ctx_t*)h)->level_start, sizeof(uint32_t) * 12);
}

/* canonical table: one row per node, level-major, Morton order per level */
PSO_API void pso_tree(void* h, int32_t* depth, uint32_t* start,
                      uint32_t* count, uint32_t* leaf, uint32_t* nchild,
                      int32_t* octant, uint32_t* first_child,
                      uint32_t* parent, float* geo, float* mp, float* l_m2l,
                      float* l_tot, uint32_t* m2l_cnt, uint32_t* p2p_cnt) {
    pso_ctx_t* c = (pso_ctx_t*)h;
    for (size_t k = 0; k < c->n_nodes; ++k) {
        const pso_node_t* n = &c->nodes[k];
        depth[k]       = n->depth;
        start[k]       = n->start;
        count[k]       = n->count;
        leaf[k]        = pso_is_leaf(n);
        nchild[k]      = n->nchild;
        octant[k]      = n->octant;
        first_child[k] = n->first_child;
        parent[k]      = n->parent;
        geo[4 * k + 0] = n->x;
        geo[4 * k + 1] = n->y;
        geo[4 * k + 2] = n->z;
        geo[4 * k + 3] = n->hw;
        for (int a = 0; a < 4; ++a) {
            mp[4 * k + a]    = n->mp[a];
            l_m2l[4 * k + a] = n->l_m2l[a];
            l_tot[4 * k + a] = n->l_tot[a];
        }
        m2l_cnt[k] = n->m2l_cnt;
        p2p_cnt[k] = n->p2p_cnt;
    }
}

PSO_API void pso_p2p_list(void* h, uint32_t* t, uint32_t* s) {
    pso_ctx_t* c = (pso_ctx_t*)h;
    memcpy(t, c->p2p_t, c->n_p2p * sizeof(uint32_t));
    memcpy(s, c->p2p_s, c->n_p2p * sizeof(uint32_t));
}

/* ---------------------------------------------------------------------
 * FP64 direct sum (tests/accuracy.c:42-72): F_i = sum_{j != i} m_i m_j d /
 * (|d|^2 + eps2)^{3/2}, for the targets listed in `targets` (all if NULL).
 * eps2 is the float literal 0.1F widened to double, as in accuracy.c:12,57.
 * ------------------------------------------------------------------- */
PSO_API void pso_direct_f64(size_t n, const float* x, const float* y,
                            const float* z, const float* m,
                            const uint32_t* targets, size_t n_targets,
                            double* fx, double* fy, double* fz) {
    size_t nt = targets ? n_targets : n;
    for (size_t k = 0; k < nt; ++k) {
        size_t i  = targets ? targets[k] : k;
        double ax = 0.0, ay = 0.0, az = 0.0;
        for (size_t j = 0; j < n; ++j) {
            if (i == j) {
                continue;
            }
            double dx    = (double)x[j] - (double)x[i];
            double dy    = (double)y[j] - (double)y[i];
            double dz    = (double)z[j] - (double)z[i];
            double r2    = (dx * dx) + (dy * dy) + (dz * dz) + (double)0.1F;
            double ir    = 1.0 / sqrt(r2);
            double ir3   = ir * ir * ir;
            double scale = (double)m[i] * (double)m[j] * ir3;
            ax += dx * scale;
            ay += dy * scale;
            az += dz * scale;
        }
        fx[k] = ax;
        fy[k] = ay;
        fz[k] = az;
    }
}

/* ---------------------------------------------------------------------
 * The caller's update after a tick (README.md:82-111, demo/unary.c:
 * 146-184): velocities permuted through ids (v_new[i] = v[ids[i]]), then
 * semi-implicit Euler for particles with positive mass.  vtmp holds 3 x n
 * floats of scratch.
 * ------------------------------------------------------------------- */
PSO_API void pso_euler_step(size_t n, const uint32_t* ids, float* vx, float* vy,
                            float* vz, float* x, float* y, float* z,
                            const float* m, const float* fx, const float* fy,
                            const float* fz, float dt, float* vtmp) {
    for (size_t i = 0; i < n; ++i) {
        uint32_t old   = ids[i];
        vtmp[i]        = vx[old];
        vtmp[n + i]    = vy[old];
        vtmp[2 * n + i] = vz[old];
    }
    for (size_t i = 0; i < n; ++i) {
        vx[i] = vtmp[i];
        vy[i] = vtmp[n + i];
        vz[i] = vtmp[2 * n + i];
    }
    for (size_t i = 0; i < n; ++i) {
        if (m[i] <= 0.0F) {
            continue;
        }
        vx[i] += (fx[i] / m[i]) * dt;
        vy[i] += (fy[i] / m[i]) * dt;
        vz[i] += (fz[i] / m[i]) * dt;
        x[i] += vx[i] * dt;
        y[i] += vy[i] * dt;
        z[i] += vz[i] * dt;
    }
}

/* ---------------------------------------------------------------------
 * Single-pass helpers mirroring the hand-built node tests of the reference
 * (tests/main.c:235-476, tests/accuracy.c:74-109).
 * ------------------------------------------------------------------- */

/* P2M of one leaf centred at (cx, cy, cz) (polesitter.h:978-1004) */
PSO_API void pso_p2m(size_t n, const float* x, const float* y, const float* z,
                     const float* m, float cx, float cy, float cz, float* out4) {
    pso_node_t nd;
    memset(&nd, 0, sizeof(nd));
    nd.x = cx;
    nd.y = cy;
    nd.z = cz;
    nd.count = (uint32_t)n;
    pso_ctx_t c;
    memset(&c, 0, sizeof(c));
    c.x = x;
    c.y = y;
    c.z = z;
    c.m = m;
    c.nodes = &nd;
    c.n_nodes = 1;
    pso_upward(&c);
    memcpy(out4, nd.mp, sizeof(nd.mp));
}

/* one MAC + M2L step on a (target, source) pair of leaves
 * (polesitter.h:1056-1094); returns 1 when the pair was separated */
PSO_API int pso_m2l_pair(const float* tgt_geo, const float* src_geo,
                         const float* src_mp, float theta, float* out_local) {
    pso_node_t nodes[2];
    memset(nodes, 0, sizeof(nodes));
    nodes[0].x = tgt_geo[0];
    nodes[0].y = tgt_geo[1];
    nodes[0].z = tgt_geo[2];
    nodes[0].hw = tgt_geo[3];
    nodes[1].x = src_geo[0];
    nodes[1].y = src_geo[1];
    nodes[1].z = src_geo[2];
    nodes[1].hw = src_geo[3];
    memcpy(nodes[1].mp, src_mp, 4 * sizeof(float));
    pso_ctx_t c;
    memset(&c, 0, sizeof(c));
    c.nodes = nodes;
    c.n_nodes = 2;
    c.theta = theta;
    pso_interact(&c, 0, 1);
    free(c.p2p_t);
    free(c.p2p_s);
    memcpy(out_local, nodes[0].l_m2l, 4 * sizeof(float));
    return nodes[0].m2l_cnt > 0;
}

/* direct leaf x leaf sum of particles [t0, t0+tn) from [s0, s0+sn)
 * (polesitter.h:1279-1449), accumulated into fx, fy, fz */
PSO_API void pso_p2p_pair(const float* x, const float* y, const float* z,
                          const float* m, float* fx, float* fy, float* fz,
                          uint32_t t0, uint32_t tn, uint32_t s0, uint32_t sn) {
    pso_node_t nodes[2];
    memset(nodes, 0, sizeof(nodes));
    nodes[0].start = t0;
    nodes[0].count = tn;
    nodes[1].start = s0;
    nodes[1].count = sn;
    pso_ctx_t c;
    memset(&c, 0, sizeof(c));
    c.x = x;
    c.y = y;
    c.z = z;
    c.m = m;
    pso_p2p_leaves(&c, &nodes[0], &nodes[1], fx, fy, fz);
}
