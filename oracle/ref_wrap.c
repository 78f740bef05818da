/*
 * Test-only wrapper that compiles the UNMODIFIED polesitter single header
 * (src/polesitter.h, included from the reference checkout by include path,
 * never copied) into oracle/_ref/libpsref*.so.
 *
 * The reference's public functions are renamed here with a psref_ prefix and
 * everything else is hidden, so this library can be loaded next to
 * libpolesitter_b200.so (which exports the real ps_* names) in one process.
 *
 * Besides the four public calls it exports white-box views that the
 * reference's own unit tests use (tests/main.c includes the header for the
 * same reason): the tree after a tick, flattened into a canonical level-major
 * Morton-ordered table, and single-pair drivers for the static M2L / P2P /
 * MAC code so the oracle can be checked against the reference's compiled
 * arithmetic on hand-made node pairs.
 *
 * This is the checker's build, not product code.  It is built by
 * oracle/build_ref.sh with the reference's own CMake flags
 * (CMakeLists.txt:37-46) plus PS_MULTITHREADING, which every reference test
 * and benchmark defines (tests/main.c:7-9).
 */
#define PS_MULTITHREADING
#define POLESITTER_IMPLEMENTATION
#include "polesitter.h"

#include <stdlib.h>

#define PSREF_API __attribute__((visibility("default")))

PSREF_API size_t psref_ctx_size(void) { return sizeof(ps_context_t); }

PSREF_API int psref_init(ps_context_t** out_ctx, const ps_config_t* cfg) {
    return (int)ps_init(out_ctx, cfg);
}

PSREF_API int psref_prepare(ps_particle_arrs_t* arrs, uint32_t* codes,
                            float* mn, float* mx, float* range) {
    return (int)ps_prepare_particles(arrs, codes, mn, mx, range);
}

PSREF_API int psref_calc(ps_context_t* ctx, const ps_particle_arrs_t* arrs,
                         uint32_t* codes, float cx, float cy, float cz,
                         float hw) {
    return (int)ps_calc_forces(ctx, arrs, codes, cx, cy, cz, hw);
}

PSREF_API int psref_destroy(ps_context_t* ctx) { return (int)ps_destroy(ctx); }

PSREF_API uint32_t psref_morton_encode(uint32_t x, uint32_t y, uint32_t z) {
    return ps_impl_morton_encode(x, y, z);
}

/* ---- tree view after a tick ------------------------------------------- */

static size_t count_rec(ps_context_t* ctx, ps_node_t* n) {
    if (!n) {
        return 0;
    }
    size_t c = 1;
    if (!(n->data.leaf.is_leaf & 1)) {
        for (int i = 0; i < 8; ++i) {
            c += count_rec(ctx, ps_impl_get_node(ctx, n->data.children_offs[i]));
        }
    }
    return c;
}

PSREF_API size_t psref_tree_nodes(ps_context_t* ctx) {
    return count_rec(ctx, ctx->root);
}

/* Breadth-first walk in child (octant) order: this lists every level in
 * Morton order, which is the canonical layout both the oracle and the GPU
 * tree use.  Per node: depth, first particle, particle count, leaf flag,
 * child count, octant digit, (x, y, z, half_width), multipole[4],
 * local_exp[4].  Returns the number of nodes written (<= cap). */
PSREF_API size_t psref_tree_dump(ps_context_t* ctx, size_t cap, int32_t* depth,
                                 uint32_t* start, uint32_t* count,
                                 uint32_t* leaf, uint32_t* nchild,
                                 int32_t* octant, float* geo, float* mp,
                                 float* loc) {
    size_t total = psref_tree_nodes(ctx);
    if (total > cap) {
        return 0;
    }
    ps_node_t** q  = (ps_node_t**)malloc(total * sizeof(ps_node_t*));
    int32_t*    dq = (int32_t*)malloc(total * sizeof(int32_t));
    int32_t*    oq = (int32_t*)malloc(total * sizeof(int32_t));
    size_t      hd = 0;
    size_t      tl = 0;
    q[tl]          = ctx->root;
    dq[tl]         = 0;
    oq[tl]         = -1;
    ++tl;
    while (hd < tl) {
        ps_node_t* n = q[hd];
        size_t     k = hd;
        depth[k]     = dq[hd];
        octant[k]    = oq[hd];
        geo[(4 * k) + 0] = n->x;
        geo[(4 * k) + 1] = n->y;
        geo[(4 * k) + 2] = n->z;
        geo[(4 * k) + 3] = n->half_width;
        float* l         = ps_impl_get_local(ctx, n);
        for (int i = 0; i < 4; ++i) {
            mp[(4 * k) + i]  = n->multipole[i];
            loc[(4 * k) + i] = l[i];
        }
        if (n->data.leaf.is_leaf & 1) {
            leaf[k]   = 1;
            start[k]  = n->data.leaf.first_particle_idx;
            count[k]  = n->data.leaf.particle_cnt;
            nchild[k] = 0;
        } else {
            leaf[k]   = 0;
            nchild[k] = 0;
            start[k]  = 0xFFFFFFFFu;
            count[k]  = 0;
            for (int i = 0; i < 8; ++i) {
                ps_node_t* c = ps_impl_get_node(ctx, n->data.children_offs[i]);
                if (!c) {
                    continue;
                }
                q[tl]  = c;
                dq[tl] = dq[hd] + 1;
                oq[tl] = i;
                ++tl;
                ++nchild[k];
            }
        }
        ++hd;
    }
    /* internal nodes: derive [start, start+count) from the leaves below, in
     * reverse BFS order so children are final before their parent. */
    /* children of node k are contiguous in BFS order; recover them by a
     * second pass that records each node's first child index. */
    size_t* first_child = (size_t*)malloc(total * sizeof(size_t));
    size_t  next        = 1;
    for (size_t k = 0; k < total; ++k) {
        first_child[k] = next;
        next += nchild[k];
    }
    for (size_t kk = total; kk-- > 0;) {
        if (leaf[kk]) {
            continue;
        }
        uint32_t s = 0xFFFFFFFFu;
        uint32_t c = 0;
        for (size_t j = 0; j < nchild[kk]; ++j) {
            size_t ch = first_child[kk] + j;
            if (start[ch] < s) {
                s = start[ch];
            }
            c += count[ch];
        }
        start[kk] = s;
        count[kk] = c;
    }
    free(first_child);
    free(q);
    free(dq);
    free(oq);
    return total;
}

/* ---- single-pair drivers over the static passes ------------------------ */

static void* g_pair_buf = NULL;

static ps_context_t* pair_ctx(float theta) {
    const size_t sz = 1u << 20;
    if (!g_pair_buf) {
        g_pair_buf = malloc(sz);
    }
    ps_context_t* ctx = NULL;
    ps_config_t   cfg = {g_pair_buf, sz, 16, theta, 1};
    ps_init(&ctx, &cfg);
    ps_impl_arena_clear(&ctx->arena);
    return ctx;
}

/* One interaction-pass call on a (target, source) pair of hand-built nodes
 * (both marked as leaves so the pass never recurses).  Writes the target's
 * local expansion and returns 1 if the MAC accepted the pair (M2L applied). */
PSREF_API int psref_m2l_pair(const float* tgt_geo, const float* src_geo,
                             const float* src_mp, float theta, float* out_loc) {
    ps_context_t* ctx = pair_ctx(theta);
    ps_node_t*    t   = ps_impl_alloc_node(ctx);
    ps_node_t*    s   = ps_impl_alloc_node(ctx);
    t->x = tgt_geo[0];
    t->y = tgt_geo[1];
    t->z = tgt_geo[2];
    t->half_width = tgt_geo[3];
    s->x = src_geo[0];
    s->y = src_geo[1];
    s->z = src_geo[2];
    s->half_width = src_geo[3];
    for (int i = 0; i < 4; ++i) {
        s->multipole[i] = src_mp[i];
    }
    t->data.leaf.is_leaf = 1;
    s->data.leaf.is_leaf = 1;
    ps_impl_fmm_interaction_pass(ctx, t, s, ctx->theta);
    float* l = ps_impl_get_local(ctx, t);
    int    hit = 0;
    for (int i = 0; i < 4; ++i) {
        out_loc[i] = l[i];
        hit |= (l[i] != 0.0F);
    }
    ps_destroy(ctx);
    return hit;
}

/* P2P between two hand-built leaves over caller arrays (target forces are
 * accumulated into fx/fy/fz exactly as the reference's leaf x leaf loop). */
PSREF_API void psref_p2p_pair(const ps_particle_arrs_t* arrs, uint32_t t_first,
                              uint32_t t_cnt, uint32_t s_first, uint32_t s_cnt) {
    ps_context_t* ctx = pair_ctx(1.0F);
    ps_node_t*    t   = ps_impl_alloc_node(ctx);
    ps_node_t*    s   = ps_impl_alloc_node(ctx);
    t->data.leaf.is_leaf            = 1;
    t->data.leaf.first_particle_idx = t_first;
    t->data.leaf.particle_cnt       = t_cnt;
    s->data.leaf.is_leaf            = 1;
    s->data.leaf.first_particle_idx = s_first;
    s->data.leaf.particle_cnt       = s_cnt;
    /* identical centres and a huge half width: never well separated */
    t->half_width = 1e10F;
    s->half_width = 1e10F;
    ps_impl_fmm_p2p_pass(ctx, t, s, arrs, ctx->theta);
    ps_destroy(ctx);
}
