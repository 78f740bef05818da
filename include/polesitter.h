/*
 * polesitter.h -- drop-in public API of the B200 FMM tick.
 *
 * Declares exactly the interface of the reference single header
 * (src/polesitter.h:290-341) so that code written against polesitter links
 * against libpolesitter_b200.so instead of defining
 * POLESITTER_IMPLEMENTATION:
 *
 *   ps_result_t    polesitter.h:294-300  (same enumerators and values; one
 *                                         value appended: PS_EDEVICE)
 *   ps_config_t    polesitter.h:304-310  (same fields, same meaning)
 *   ps_particle_arrs_t polesitter.h:312-322 (same fields; each array may be
 *                                         host memory or CUDA device memory)
 *   ps_init              replaces polesitter.h:325 / :1699-1767
 *   ps_calc_forces       replaces polesitter.h:328-330 / :1840-1909
 *   ps_prepare_particles replaces polesitter.h:334-336 / :1911-2170
 *   ps_destroy           replaces polesitter.h:339 / :2172-2192
 *
 * Behaviour kept from the reference: the context lives inside cfg->buff;
 * ps_calc_forces sorts x, y, z, mass, id and the Morton codes in place by
 * code (stable), permutes ids along, zeroes and then writes fx, fy, fz in the
 * sorted order; ps_prepare_particles takes no context and returns the cubic
 * bounding box; theta <= 0 selects 1.0; thrd_cnt is accepted (the GPU grid
 * replaces the thread pool).  Differences: device scratch is cudaMalloc'ed
 * by ps_init (sized from max_particles) and freed by ps_destroy; a count
 * above max_particles is rejected with PS_EINVAL instead of overrunning.
 */
#ifndef POLESITTER_H
#define POLESITTER_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    PS_OK = 0,
    PS_EOOM = -1,    /* out of memory */
    PS_EINVAL = -2,  /* invalid argument */
    PS_ETHRD = -3,   /* thread creation failed (kept for ABI; not produced) */
    PS_EALLOC = -4,  /* allocation failed (device memory) */
    PS_EDEVICE = -5, /* CUDA runtime / device status error */
} ps_result_t;

typedef struct ps_context ps_context_t;

typedef struct {
    void* buff;           /* host memory provided by the caller */
    size_t buff_size;     /* total size in bytes */
    size_t max_particles; /* maximum particle count of a tick */
    float theta;          /* MAC threshold; 0.0F defaults to 1.0F */
    size_t thrd_cnt;      /* accepted for compatibility; unused */
} ps_config_t;

typedef struct {
    float* x;
    float* y;
    float* z;
    float* mass;
    float* fx;
    float* fy;
    float* fz;
    uint32_t* id;
    size_t cnt;
} ps_particle_arrs_t;

/* init pipeline with a pre-allocated buffer */
ps_result_t ps_init(ps_context_t** out_ctx, const ps_config_t* cfg);

/* compute forces on particles using FMM */
ps_result_t ps_calc_forces(ps_context_t* ctx, const ps_particle_arrs_t* arrs,
                           uint32_t* morton_codes, float root_cx, float root_cy,
                           float root_cz, float root_hw);

/* calculates the global bounding box and generates morton codes for all
 * particles */
ps_result_t ps_prepare_particles(ps_particle_arrs_t* arrs, uint32_t* out_morton_codes,
                                 float* out_min_b, float* out_max_b, float* out_range);

/* releases the context's device resources */
ps_result_t ps_destroy(ps_context_t* ctx);

#ifdef __cplusplus
}
#endif

#endif /* POLESITTER_H */
