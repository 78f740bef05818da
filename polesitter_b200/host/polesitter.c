/*
 * Host layer of libpolesitter_b200.so (C99): argument checks and the context
 * layout of the reference's public API, over the CUDA shim declared in
 * csrc/psg_internal.h.
 *
 * Each function keeps the reference's argument meaning and error results:
 *   ps_init              polesitter.h:1699-1767
 *   ps_prepare_particles polesitter.h:1911-2170
 *   ps_calc_forces       polesitter.h:1840-1909
 *   ps_destroy           polesitter.h:2172-2192
 */
#include <stdint.h>
#include <string.h>

#include "../../include/polesitter.h"
#include "../../include/polesitter_b200.h"
#include "../csrc/psg_internal.h"

#define PS_CTX_MAGIC 0x70736232u /* "psb2" */

/* The context sits at the start of cfg->buff like the reference's
 * (polesitter.h:1705); the device-side state follows at a 64-byte offset. */
struct ps_context {
    uint32_t magic;
    uint32_t reserved;
    float theta;
    size_t max_particles;
    size_t thrd_cnt;
};

#define PS_CTX_HDR 64u

static int g_morton_variant = PSG_MORTON_AVX2;

static size_t align64(size_t v) { return (v + 63u) & ~(size_t)63u; }

static void* ctx_state(ps_context_t* ctx) { return (uint8_t*)ctx + PS_CTX_HDR; }

size_t ps_b200_context_size(void) { return PS_CTX_HDR + psg_state_bytes(); }

static ps_result_t to_ps(int r) { return (ps_result_t)r; }

ps_result_t ps_init(ps_context_t** out_ctx, const ps_config_t* cfg) {
    if (!out_ctx || !cfg || !cfg->buff || cfg->buff_size < ps_b200_context_size()) {
        return PS_EINVAL; /* polesitter.h:1700 */
    }
    /* the reference reserves 6 x 4 B per particle of radix temporaries at
     * the buffer end and fails with PS_EOOM when they do not fit
     * (:1716-1723); the same sizing rule is kept so callers see the same
     * result for the same buffer */
    size_t radix_tmp = 6u * cfg->max_particles * sizeof(float);
    if (align64(ps_b200_context_size()) + radix_tmp > cfg->buff_size) {
        return PS_EOOM;
    }
    if (cfg->max_particles > (size_t)60000000u) {
        return PS_EINVAL; /* node ids are packed in 28 bits in the traversal */
    }
    ps_context_t* ctx = (ps_context_t*)cfg->buff;
    memset(ctx, 0, PS_CTX_HDR);
    ctx->theta = (cfg->theta > 0.0F) ? cfg->theta : 1.0F; /* :1707 */
    ctx->max_particles = cfg->max_particles;
    ctx->thrd_cnt = cfg->thrd_cnt;
    int r = psg_init(ctx_state(ctx), cfg->max_particles, ctx->theta);
    if (r != PSG_OK) {
        return to_ps(r);
    }
    ctx->magic = PS_CTX_MAGIC;
    *out_ctx = ctx;
    return PS_OK;
}

ps_result_t ps_prepare_particles(ps_particle_arrs_t* arrs, uint32_t* out_morton_codes,
                                 float* out_min_b, float* out_max_b, float* out_range) {
    if (!arrs || !out_morton_codes || arrs->cnt == 0) {
        return PS_EINVAL; /* :1914 */
    }
    if (!arrs->x || !arrs->y || !arrs->z) {
        return PS_EINVAL;
    }
    psg_arrays_t a;
    memset(&a, 0, sizeof(a));
    a.x = arrs->x;
    a.y = arrs->y;
    a.z = arrs->z;
    a.codes = out_morton_codes;
    a.n = arrs->cnt;
    return to_ps(psg_prepare(&a, out_min_b, out_max_b, out_range, g_morton_variant));
}

ps_result_t ps_calc_forces(ps_context_t* ctx, const ps_particle_arrs_t* arrs,
                           uint32_t* morton_codes, float root_cx, float root_cy,
                           float root_cz, float root_hw) {
    if (!ctx || !arrs || ctx->magic != PS_CTX_MAGIC) {
        return PS_EINVAL; /* :1843 */
    }
    if (arrs->cnt == 0) {
        return PS_OK; /* nothing to sort, no forces (:1592-1594) */
    }
    if (!morton_codes || !arrs->x || !arrs->y || !arrs->z || !arrs->mass || !arrs->fx ||
        !arrs->fy || !arrs->fz || !arrs->id) {
        return PS_EINVAL;
    }
    psg_arrays_t a;
    a.x = arrs->x;
    a.y = arrs->y;
    a.z = arrs->z;
    a.mass = arrs->mass;
    a.fx = arrs->fx;
    a.fy = arrs->fy;
    a.fz = arrs->fz;
    a.id = arrs->id;
    a.codes = morton_codes;
    a.n = arrs->cnt;
    return to_ps(psg_calc(ctx_state(ctx), &a, root_cx, root_cy, root_cz, root_hw));
}

ps_result_t ps_destroy(ps_context_t* ctx) {
    if (!ctx || ctx->magic != PS_CTX_MAGIC) {
        return PS_EINVAL; /* :2173 */
    }
    int r = psg_destroy(ctx_state(ctx));
    ctx->magic = 0;
    return to_ps(r);
}

/* ---- extensions (include/polesitter_b200.h) ---------------------------- */

ps_result_t ps_b200_set_option(ps_context_t* ctx, int key, double value) {
    if (!ctx || ctx->magic != PS_CTX_MAGIC) {
        return PS_EINVAL;
    }
    if (key == PS_B200_OPT_THETA) {
        ctx->theta = value > 0.0 ? (float)value : 1.0F;
    }
    return to_ps(psg_set_option(ctx_state(ctx), key, value));
}

ps_result_t ps_b200_set_morton_variant(int variant) {
    if (variant < PSG_MORTON_AVX2 || variant > PSG_MORTON_SCALAR) {
        return PS_EINVAL;
    }
    g_morton_variant = variant;
    return PS_OK;
}

ps_result_t ps_b200_get_stats(ps_context_t* ctx, uint64_t* out, size_t n) {
    if (!ctx || ctx->magic != PS_CTX_MAGIC) {
        return PS_EINVAL;
    }
    return to_ps(psg_get_stats(ctx_state(ctx), out, n));
}

ps_result_t ps_b200_last_timing(ps_context_t* ctx, float* ms, size_t n) {
    if (!ctx || ctx->magic != PS_CTX_MAGIC) {
        return PS_EINVAL;
    }
    return to_ps(psg_last_timing(ctx_state(ctx), ms, n));
}

size_t ps_b200_tree_nodes(ps_context_t* ctx) {
    if (!ctx || ctx->magic != PS_CTX_MAGIC) {
        return 0;
    }
    return psg_tree_nodes(ctx_state(ctx));
}

ps_result_t ps_b200_tree_dump(ps_context_t* ctx, size_t cap, int32_t* depth, uint32_t* start,
                              uint32_t* count, uint32_t* nchild, int32_t* octant,
                              uint32_t* first_child, uint32_t* parent, float* geo, float* mp,
                              float* local_exp, uint32_t* m2l_cnt, uint32_t* p2p_cnt) {
    if (!ctx || ctx->magic != PS_CTX_MAGIC) {
        return PS_EINVAL;
    }
    return to_ps(psg_tree_dump(ctx_state(ctx), cap, depth, start, count, nchild, octant,
                               first_child, parent, geo, mp, local_exp, m2l_cnt, p2p_cnt));
}

ps_result_t ps_b200_direct_f64(ps_context_t* ctx, const ps_particle_arrs_t* arrs,
                               const uint32_t* targets, size_t n_targets, double* out) {
    if (!ctx || ctx->magic != PS_CTX_MAGIC || !arrs) {
        return PS_EINVAL;
    }
    psg_arrays_t a;
    memset(&a, 0, sizeof(a));
    a.x = arrs->x;
    a.y = arrs->y;
    a.z = arrs->z;
    a.mass = arrs->mass;
    a.n = arrs->cnt;
    return to_ps(psg_direct_f64(ctx_state(ctx), &a, targets, n_targets, out));
}

ps_result_t ps_b200_run_ticks(ps_context_t* ctx, const ps_particle_arrs_t* arrs,
                              uint32_t* morton_codes, float* vx, float* vy, float* vz,
                              float dt, uint32_t ticks) {
    if (!ctx || !arrs || ctx->magic != PS_CTX_MAGIC) {
        return PS_EINVAL;
    }
    if (arrs->cnt == 0 || ticks == 0) {
        return PS_OK;
    }
    if (!morton_codes || !arrs->x || !arrs->y || !arrs->z || !arrs->mass || !arrs->fx ||
        !arrs->fy || !arrs->fz || !arrs->id || !vx || !vy || !vz) {
        return PS_EINVAL;
    }
    psg_arrays_t a;
    a.x = arrs->x;
    a.y = arrs->y;
    a.z = arrs->z;
    a.mass = arrs->mass;
    a.fx = arrs->fx;
    a.fy = arrs->fy;
    a.fz = arrs->fz;
    a.id = arrs->id;
    a.codes = morton_codes;
    a.n = arrs->cnt;
    return to_ps(psg_run_ticks(ctx_state(ctx), &a, vx, vy, vz, dt, ticks, g_morton_variant));
}

#define PS_CTX_OK(ctx) ((ctx) && (ctx)->magic == PS_CTX_MAGIC)

ps_result_t ps_b200_closure_set_weights(ps_context_t* ctx, const float* params, size_t n) {
    if (!PS_CTX_OK(ctx) || !params) {
        return PS_EINVAL;
    }
    return to_ps(psg_closure_set_weights(ctx_state(ctx), params, n));
}

ps_result_t ps_b200_closure_last(ps_context_t* ctx, double* median_base, double* median_mlp,
                                 int* used, int* samples) {
    if (!PS_CTX_OK(ctx)) {
        return PS_EINVAL;
    }
    return to_ps(psg_closure_last(ctx_state(ctx), median_base, median_mlp, used, samples));
}

ps_result_t ps_b200_closure_features(ps_context_t* ctx, const uint32_t* idx, size_t k,
                                     float* x_out, float* scale_out) {
    if (!PS_CTX_OK(ctx)) {
        return PS_EINVAL;
    }
    return to_ps(psg_closure_features(ctx_state(ctx), idx, k, x_out, scale_out));
}

ps_result_t ps_b200_closure_correction(ps_context_t* ctx, float* out, size_t n) {
    if (!PS_CTX_OK(ctx)) {
        return PS_EINVAL;
    }
    return to_ps(psg_closure_correction(ctx_state(ctx), out, n));
}

ps_result_t ps_b200_closure_forward(ps_context_t* ctx, const float* x, size_t n,
                                    const float* params, float* y_out) {
    if (!PS_CTX_OK(ctx)) {
        return PS_EINVAL;
    }
    return to_ps(psg_closure_forward(ctx_state(ctx), x, n, params, y_out));
}

ps_result_t ps_b200_closure_grad(ps_context_t* ctx, const float* x, const float* t, size_t n,
                                 const float* params, float* grad_out, float* loss_out) {
    if (!PS_CTX_OK(ctx)) {
        return PS_EINVAL;
    }
    return to_ps(psg_closure_grad(ctx_state(ctx), x, t, n, params, grad_out, loss_out));
}

ps_result_t ps_b200_closure_train(ps_context_t* ctx, const float* x, const float* t, size_t n,
                                  float* params, uint32_t epochs, uint32_t batch, float lr,
                                  uint64_t seed, float* loss_out) {
    if (!PS_CTX_OK(ctx)) {
        return PS_EINVAL;
    }
    return to_ps(psg_closure_train(ctx_state(ctx), x, t, n, params, epochs, batch, lr, seed,
                                   loss_out));
}

static void ens_arrays(psg_arrays_t* a, const ps_particle_arrs_t* arrs, uint32_t* codes) {
    a->x = arrs->x;
    a->y = arrs->y;
    a->z = arrs->z;
    a->mass = arrs->mass;
    a->fx = arrs->fx;
    a->fy = arrs->fy;
    a->fz = arrs->fz;
    a->id = arrs->id;
    a->codes = codes;
    a->n = arrs->cnt;
}

ps_result_t ps_b200_ensemble_create(ps_b200_ensemble_t** out, const size_t* counts,
                                    size_t n_systems, const float* theta) {
    if (!out) {
        return PS_EINVAL;
    }
    void* h = NULL;
    int r = psg_ensemble_create(&h, counts, n_systems, theta);
    if (r == PSG_OK) {
        *out = (ps_b200_ensemble_t*)h;
    }
    return to_ps(r);
}

ps_result_t ps_b200_ensemble_autotune(ps_b200_ensemble_t* ens, const ps_particle_arrs_t* arrs,
                                      uint32_t* morton_codes, float target_median_error,
                                      float* theta_out, double* grid_scale_out) {
    if (!ens || !arrs || !morton_codes) {
        return PS_EINVAL;
    }
    psg_arrays_t a;
    ens_arrays(&a, arrs, morton_codes);
    return to_ps(psg_ensemble_autotune(ens, &a, target_median_error, theta_out, grid_scale_out));
}

ps_result_t ps_b200_ensemble_run(ps_b200_ensemble_t* ens, const ps_particle_arrs_t* arrs,
                                 uint32_t* morton_codes, float* vx, float* vy, float* vz,
                                 float dt, uint32_t ticks) {
    if (!ens || !arrs || !morton_codes) {
        return PS_EINVAL;
    }
    psg_arrays_t a;
    ens_arrays(&a, arrs, morton_codes);
    return to_ps(psg_ensemble_run(ens, &a, vx, vy, vz, dt, ticks));
}

ps_result_t ps_b200_ensemble_theta(ps_b200_ensemble_t* ens, float* theta_out, size_t n) {
    if (!ens) {
        return PS_EINVAL;
    }
    return to_ps(psg_ensemble_systems(ens, theta_out, n));
}

ps_result_t ps_b200_ensemble_leaf_caps(ps_b200_ensemble_t* ens, uint32_t* cap_out, size_t n) {
    if (!ens) {
        return PS_EINVAL;
    }
    return to_ps(psg_ensemble_leaf_caps(ens, cap_out, n));
}

ps_result_t ps_b200_ensemble_set_leaf_caps(ps_b200_ensemble_t* ens, const uint32_t* caps,
                                           size_t n) {
    if (!ens) {
        return PS_EINVAL;
    }
    return to_ps(psg_ensemble_set_leaf_caps(ens, caps, n, 0));
}

ps_result_t ps_b200_ensemble_set_leaf_ladder(ps_b200_ensemble_t* ens, const uint32_t* caps,
                                             size_t n) {
    if (!ens) {
        return PS_EINVAL;
    }
    return to_ps(psg_ensemble_set_leaf_caps(ens, caps, n, 1));
}

ps_result_t ps_b200_ensemble_set_order(ps_b200_ensemble_t* ens, int order) {
    if (!ens) {
        return PS_EINVAL;
    }
    return to_ps(psg_ensemble_set_order(ens, order));
}

ps_result_t ps_b200_ensemble_order(ps_b200_ensemble_t* ens, int* order_out) {
    if (!ens || !order_out) {
        return PS_EINVAL;
    }
    return to_ps(psg_ensemble_order(ens, order_out));
}

ps_result_t ps_b200_ensemble_destroy(ps_b200_ensemble_t* ens) {
    if (!ens) {
        return PS_EINVAL;
    }
    return to_ps(psg_ensemble_destroy(ens));
}

const char* ps_b200_last_error(void) { return psg_last_error(); }

ps_result_t ps_b200_prepare_particles_noalloc(ps_particle_arrs_t* arrs,
                                              uint32_t* out_morton_codes, float* out_min_b,
                                              float* out_max_b, float* out_range) {
    if (!arrs || !out_morton_codes || arrs->cnt == 0) {
        psg_set_error("ps_b200_prepare_particles_noalloc: null argument or zero count");
        return PS_EINVAL;
    }
    return to_ps(psg_prepare_noalloc(arrs->x, arrs->y, arrs->z, arrs->cnt, out_morton_codes,
                                     out_min_b, out_max_b, out_range, g_morton_variant));
}
