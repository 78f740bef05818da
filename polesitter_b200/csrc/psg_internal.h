/*
 * Internal C ABI between the C99 host layer (host/polesitter.c) and the CUDA
 * side of libpolesitter_b200.so.  Plain pointers and sizes only.
 */
#ifndef PSG_INTERNAL_H
#define PSG_INTERNAL_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* result codes: the reference's ps_result_t values (polesitter.h:294-300)
 * plus one for a CUDA runtime failure */
#define PSG_OK 0
#define PSG_EOOM (-1)
#define PSG_EINVAL (-2)
#define PSG_ETHRD (-3)
#define PSG_EALLOC (-4)
#define PSG_EDEVICE (-5)

/* device status error bits */
#define PSG_ERR_SORT_SPIN 0x1u    /* a look-back wait ran out of iterations */
#define PSG_ERR_NS_OVERFLOW 0x2u  /* near-list region too small: regrow, rerun */
#define PSG_ERR_STACK 0x4u        /* traversal stack bound violated */
#define PSG_ERR_NODES 0x8u        /* tree level over its capacity */
#define PSG_ERR_P2P_OVERFLOW 0x10u /* P2P chunk store too small: regrow, rerun */
#define PSG_ERR_DENSE_OVERFLOW 0x20u /* full-leaf record list too small: regrow, rerun */
#define PSG_ERR_HEAVY_OVERFLOW 0x40u /* shallow-leaf records or frontier too small */
#define PSG_ERR_CHAIN_ORDER 0x80u   /* an order-1 group without near lists (host bug) */
#define PSG_ERR_TC_TIMEOUT 0x100u   /* a tensor-core MMA did not complete in time */

/* debug statistics slots (Status.stat) */
#define PSG_STAT_MAC 0
#define PSG_STAT_M2L 1
#define PSG_STAT_P2P_PAIRS 2
#define PSG_STAT_P2P_INTER 3
#define PSG_STAT_CHUNKS_A 4     /* candidate chunks from near lists / root */
#define PSG_STAT_CHUNKS_DFS 5   /* candidate chunks from the DFS stack */
#define PSG_STAT_TESTS_A 6      /* (candidate, child) MAC tests, first pass */
#define PSG_STAT_TESTS_DFS 7    /* MAC tests inside the leaf descents */
#define PSG_STAT_LANES 8        /* occupied candidate lanes over all chunks */
#define PSG_STAT_GROUPS 9       /* groups processed (leaf mode) */
#define PSG_STAT_DFS_STEPS 10
#define PSG_STAT_SLOWEST_GROUP 11 /* leaf pass: (clock cycles << 28) | node of the slowest group */
#define PSG_STAT_DENSE_INTER 12   /* particle pairs summed by the full-leaf kernel */

/* Morton quantisation variants of polesitter.h:2013-2157 */
#define PSG_MORTON_AVX2 0
#define PSG_MORTON_NEON 1
#define PSG_MORTON_SCALAR 2

/* caller arrays for one tick; each pointer may be host or device memory */
typedef struct {
    float* x;
    float* y;
    float* z;
    float* mass;
    float* fx;
    float* fy;
    float* fz;
    uint32_t* id;
    uint32_t* codes;
    size_t n;
} psg_arrays_t;

/* bytes of host memory the device state needs (placed in the caller's
 * ps_config_t buffer right after the context header) */
size_t psg_state_bytes(void);

int psg_init(void* state, size_t max_particles, float theta);
int psg_destroy(void* state);

/* ps_prepare_particles: bbox + Morton codes.  Uses a process-wide workspace
 * on the current CUDA device. */
int psg_prepare(const psg_arrays_t* a, float* out_min, float* out_max,
                float* out_range, int morton_variant);

/* ps_calc_forces on a context */
int psg_calc(void* state, const psg_arrays_t* a, float cx, float cy, float cz,
             float hw);

/* options and introspection (extended API) */
int psg_set_option(void* state, int key, double value);
int psg_get_stats(void* state, uint64_t* out, size_t n_out);
size_t psg_tree_nodes(void* state);
int psg_tree_dump(void* state, size_t cap, int32_t* depth, uint32_t* start,
                  uint32_t* count, uint32_t* nchild, int32_t* octant,
                  uint32_t* first_child, uint32_t* parent, float* geo,
                  float* mp, float* lt, uint32_t* m2l_cnt, uint32_t* p2p_cnt);
int psg_last_timing(void* state, float* out_ms, size_t n_out);
int psg_direct_f64(void* state, const psg_arrays_t* a, const uint32_t* targets, size_t n_t,
                   double* out);
/* the caller's tick loop on the device (k_tick.cu) */
int psg_run_ticks(void* state, const psg_arrays_t* a, float* vx, float* vy, float* vz, float dt,
                  uint32_t ticks, int morton_variant);
/* batched ensemble of independent systems (CUDA graphs; psg_runtime.cu) */
int psg_ensemble_create(void** out, const size_t* counts, size_t n_systems, const float* theta);
int psg_ensemble_destroy(void* ens);
int psg_ensemble_run(void* ens, const psg_arrays_t* a, float* vx, float* vy, float* vz, float dt,
                     uint32_t ticks);
int psg_ensemble_autotune(void* ens, const psg_arrays_t* a, float target, float* theta_out,
                          double* grid_scale_out);
int psg_ensemble_systems(void* ens, float* theta_out, size_t n);
int psg_ensemble_leaf_caps(void* ens, uint32_t* cap_out, size_t n);
/* ladder != 0: the leaf capacities the autotuner tries; else one per system */
int psg_ensemble_set_leaf_caps(void* ens, const uint32_t* caps, size_t n, int ladder);
/* local expansion order of all systems (0 or 1; < 0: the autotuner tries both) */
int psg_ensemble_set_order(void* ens, int order);
int psg_ensemble_order(void* ens, int* out);
const char* psg_last_error(void);
void psg_set_error(const char* msg);

/* ps_prepare_particles with a fixed static scratch (k_noalloc.cu) */
int psg_prepare_noalloc(const float* x, const float* y, const float* z, size_t n,
                        uint32_t* codes, float* out_min, float* out_max, float* out_range,
                        int variant);

#define PSG_OPT_DEBUG 1          /* 1: record per-node interaction counts */
#define PSG_OPT_THETA 2
#define PSG_OPT_MORTON_VARIANT 3
#define PSG_OPT_TIMING 4         /* 1: time phases with CUDA events */
#define PSG_OPT_KAHAN 6          /* 1: compensated FP32 sums in P2P */
#define PSG_OPT_CLOSURE 7        /* 0 reference, 1 order-1 local, 2 + learned correction */
#define PSG_OPT_JUDGE 8          /* 1: sampled FP64 judge in closure mode 1 too */
#define PSG_OPT_HEAVY_DEPTH 9    /* leaves this shallow walk block-parallel (-1: from theta) */
#define PSG_OPT_LEAF_CAP 10      /* split nodes holding more particles than this (1..256) */
#define PSG_OPT_NEAR_LEVELS 11   /* store near lists for node depths <= this at most (2..10) */
#define PSG_OPT_STREAM 12        /* 1: sum P2P in the leaf pass, never spill it */
#define PSG_OPT_SHRINK_STORES 13 /* 1: shrink the growable traversal stores now */
#define PSG_OPT_SORT_SPIN 14     /* > 0: sort look-back polls, first tile publishing late */
#define PSG_OPT_JUDGE_BLOCKS 15  /* blocks per SM of the closure judge's FP64 sum (1..8) */
#define PSG_OPT_JUDGE_SAMPLES 16 /* particles the closure judge samples (64..4096) */
#define PSG_MAX_LEAF_CAP 256

/* the learned far-field closure (k_closure.cu) */
#define PSG_CLOSURE_PARAMS 9928
int psg_closure_set_weights(void* state, const float* params, size_t n_params);
int psg_closure_last(void* state, double* median_base, double* median_mlp, int* used,
                     int* samples);
int psg_closure_features(void* state, const uint32_t* idx, size_t k, float* x_out,
                         float* scale_out);
int psg_closure_train(void* state, const float* x, const float* t, size_t n, float* params,
                      uint32_t epochs, uint32_t batch, float lr, uint64_t seed, float* loss_out);
int psg_closure_grad(void* state, const float* x, const float* t, size_t n, const float* params,
                     float* grad_out, float* loss_out);
int psg_closure_forward(void* state, const float* x, size_t n, const float* params,
                        float* y_out);
int psg_closure_correction(void* state, float* out, size_t n);

#ifdef __cplusplus
}
#endif

#endif /* PSG_INTERNAL_H */
