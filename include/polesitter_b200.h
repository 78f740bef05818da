/*
 * polesitter_b200.h -- extensions of the drop-in API (no counterpart in the
 * reference unless stated).  Include after polesitter.h.
 */
#ifndef POLESITTER_B200_H
#define POLESITTER_B200_H

#include "polesitter.h"

#ifdef __cplusplus
extern "C" {
#endif

/* bytes of cfg->buff the context itself occupies (the reference's
 * equivalent is sizeof(ps_context_t), polesitter.h:1700) */
size_t ps_b200_context_size(void);

/* options, applied to later ticks of ctx */
#define PS_B200_OPT_DEBUG 1          /* record per-node interaction counts */
#define PS_B200_OPT_THETA 2          /* change theta after ps_init */
#define PS_B200_OPT_TIMING 4         /* time tick phases with CUDA events */
#define PS_B200_OPT_KAHAN 6          /* compensated (Kahan) FP32 sums in P2P */
#define PS_B200_OPT_CLOSURE 7        /* learned far-field closure, see below */
#define PS_B200_OPT_JUDGE 8          /* 1: run the closure's judge in mode 1 too */
#define PS_B200_OPT_HEAVY_DEPTH 9    /* leaves at most this deep (0..5) are walked by a whole
                                        block each; -1 (default): the largest d with
                                        2^d <= 4 theta */
#define PS_B200_OPT_LEAF_CAP 10      /* leaf capacity B (1..256): a node below the root
                                        holding more than B particles is split (the
                                        reference: 1, polesitter.h:911); the root is split
                                        whenever it holds 2 or more */
#define PS_B200_OPT_NEAR_LEVELS 11   /* store near lists for node depths <= this at most
                                        (2..10, default 10); leaf groups below walk their
                                        ancestor chains instead.  The library lowers it by
                                        itself when the lists would not fit (plain far field
                                        only), so every theta runs; the interaction set is
                                        the same either way */
#define PS_B200_OPT_STREAM 12        /* 1: sum each leaf group's P2P in the leaf pass as its
                                        sources are found, with no source list in device
                                        memory (chosen by the library when the lists would
                                        not fit) */
#define PS_B200_OPT_SHRINK_STORES 13 /* 1: shrink the traversal's growable stores (near
                                        lists, P2P chunks, full-leaf records) to their
                                        minimum now; the next tick grows them again */
#define PS_B200_OPT_SORT_SPIN 14     /* test of the sort's bounded wait: > 0 lets a tile's
                                        look-back poll only this many times while the first
                                        tile of the first pass publishes ~200 us late; the
                                        tick then returns PS_EDEVICE; 0 (default) restores
                                        the normal limit */
#define PS_B200_OPT_JUDGE_BLOCKS 15  /* blocks per SM (1..8, default 4) of the closure judge's
                                        FP64 direct sum, which runs beside the tree build and
                                        traversal: more take a larger share of the SMs */
#define PS_B200_OPT_JUDGE_SAMPLES 16 /* particles in the closure judge's sample (64..4096,
                                        default 1024).  Its FP64 direct sum costs samples x N
                                        pair terms a tick; the median it decides on has a
                                        relative standard error of ~1/sqrt(samples) */
ps_result_t ps_b200_set_option(ps_context_t* ctx, int key, double value);

/* Morton quantisation of ps_prepare_particles, process-wide (it takes no
 * context): 0 = AVX2 rounding (polesitter.h:2015-2073, the x86 default),
 * 1 = NEON truncation (:2074-2127), 2 = scalar (:2132-2157). */
ps_result_t ps_b200_set_morton_variant(int variant);

/* counters of the last tick: [1] M2L pairs, [2] P2P leaf pairs, [3] P2P
 * particle pairs, [9] deepest traversal stack (these need
 * PS_B200_OPT_DEBUG), [8] nodes, [10] P2P list chunks, [11] traversal runs
 * (> 1 when a capacity had to grow), [12] particles in the fullest leaf,
 * [13] full-leaf P2P work records, [14] deepest level whose near lists were
 * stored, [15] 1 when the P2P was streamed */
ps_result_t ps_b200_get_stats(ps_context_t* ctx, uint64_t* out, size_t n);

/* per-phase device times of the last tick in ms (PS_B200_OPT_TIMING):
 * [0] sort, [1] gather + write-back, [2] tree build, [3] upward pass,
 * [4] interaction pass of internal nodes (MAC/M2L/L2L, all levels),
 * [5] leaf pass (MAC/M2L/L2L + P2P + L2P), [6] whole tick, [7] learned
 * closure (correction, judge decision), [8] P2P + L2P of full leaves */
ps_result_t ps_b200_last_timing(ps_context_t* ctx, float* ms, size_t n);

/* The last tick's tree in canonical form: level-major, each level in Morton
 * order (the order the reference's recursion creates nodes,
 * polesitter.h:923-966).  Per node: depth, first particle, count, children,
 * octant, first child and parent (indices into this table), centre +
 * half-width, multipole, local expansion after the downward pass, and (with
 * PS_B200_OPT_DEBUG) the node's M2L and P2P pair counts as target. */
size_t ps_b200_tree_nodes(ps_context_t* ctx);
ps_result_t ps_b200_tree_dump(ps_context_t* ctx, size_t cap, int32_t* depth,
                              uint32_t* start, uint32_t* count, uint32_t* nchild,
                              int32_t* octant, uint32_t* first_child, uint32_t* parent,
                              float* geo, float* mp, float* local_exp,
                              uint32_t* m2l_cnt, uint32_t* p2p_cnt);

/* FP64 direct-sum forces F_i = sum_{j != i} m_i m_j d / (|d|^2 + 0.1F)^1.5
 * on the GPU (the accuracy yardstick of tests/accuracy.c:42-72) for
 * n_targets particle indices into arrs; out holds n_targets x 3 doubles.
 * Arrays may be host or device memory.  Uses ctx's device scratch, so call
 * it between ticks. */
ps_result_t ps_b200_direct_f64(ps_context_t* ctx, const ps_particle_arrs_t* arrs,
                               const uint32_t* targets, size_t n_targets, double* out);

/* ps_prepare_particles for callers that cannot allocate memory.  No
 * counterpart in the reference.  The regular ps_prepare_particles creates a
 * workspace (device buffers, a stream, a pinned buffer) on its first call;
 * callers with a fixed, pre-reserved memory budget that forbid allocation
 * inside their frame loop (so a frame never stalls on the allocator or fails
 * for want of memory) cannot let it.  This variant allocates nothing: its
 * scratch (the per-block partial bounding boxes) is a static 32 KB device
 * array loaded with the library.
 *   - arrs->x, y, z and out_morton_codes must be device memory; the three
 *     float outputs are host pointers (any may be NULL), same meaning as in
 *     ps_prepare_particles.
 *   - arrs->cnt must be 1 .. 4,194,304; larger counts return PS_EINVAL.
 *   - The first call on a device resolves the scratch's device address and
 *     keeps it for that device.  After a cudaDeviceReset that kept address
 *     is stale: do not mix this call with device resets in one process.
 *   - Runs on the legacy default stream and returns when the results are
 *     final.  All calls share the one scratch array: calls that overlap on
 *     the GPU race, so serialise them. */
ps_result_t ps_b200_prepare_particles_noalloc(ps_particle_arrs_t* arrs,
                                              uint32_t* out_morton_codes, float* out_min_b,
                                              float* out_max_b, float* out_range);

/* `ticks` iterations of the tick loop every polesitter caller writes around
 * ps_calc_forces (README.md:65-111, demo/unary.c:117-189), run without
 * leaving the device.  Each iteration:
 *   ids[i] = i; ps_prepare_particles; ps_calc_forces with the root
 *   c = min + range / 2, hw = range / 2 (README.md:76-80);
 *   v[i] = v_before[ids[i]] for vx, vy, vz (README.md:82-93);
 *   if mass[i] > 0: v += (f / m) * dt; x += v * dt (README.md:98-110).
 * On return the arrays hold the state after the last iteration: positions,
 * masses, ids and codes sorted as its calc left them, its forces, and the
 * velocities in that order.  Every step rounds as the C loop does, so a
 * loop over ps_prepare_particles + ps_calc_forces + the C update gives the
 * same positions up to the forces' own rounding.  Arrays may be host memory
 * (copied in once and out once) or device memory.  The first call
 * allocates 6 x 4 B x max_particles of velocity scratch on ctx's device. */
ps_result_t ps_b200_run_ticks(ps_context_t* ctx, const ps_particle_arrs_t* arrs,
                              uint32_t* morton_codes, float* vx, float* vy, float* vz,
                              float dt, uint32_t ticks);

/* ---- learned far-field closure (no counterpart in the reference) --------
 *
 * PS_B200_OPT_CLOSURE selects the far field of later ticks:
 *   0  the reference's (default): order-0 local expansion, additive L2L;
 *      every result is the reference's.
 *   1  order-1 local expansion: M2L also accumulates the gradient G of each
 *      monopole's field, L2L shifts the parent's field to the child's centre
 *      (L += G (c_child - c_parent)) and L2P evaluates L + G (x - c) at each
 *      particle.  Same interaction set as mode 0.
 *   2  mode 1 plus a learned correction: an MLP (16 -> 64 -> 64 -> 64 -> 8,
 *      GELU, BF16 weights, FP32 accumulation, on the tensor cores) maps each
 *      particle's leaf field, field gradient, offset in the leaf and leaf
 *      depth to a force correction.  Each tick an FP64 direct sum on a
 *      sample of particles (a new one every tick; 1024 particles unless
 *      PS_B200_OPT_JUDGE_SAMPLES says otherwise) judges it: the correction
 *      is applied only when it lowers the sample's median relative error,
 *      else the mode-1 forces stand.  Needs weights (ps_b200_closure_set_weights).
 * The parameter vector is PS_B200_CLOSURE_PARAMS floats:
 *   W1[16][64] b1[64] W2[64][64] b2[64] W3[64][64] b3[64] W4[64][8] b4[8]
 * (W[in][out]; inputs 13..15 and outputs 3..7 are padding). */
#define PS_B200_CLOSURE_PARAMS 9928
ps_result_t ps_b200_closure_set_weights(ps_context_t* ctx, const float* params, size_t n);

/* the judge of the last tick: median relative force error of the sample
 * without and with the correction, whether it was applied, sample size
 * (0 when no judge ran) */
ps_result_t ps_b200_closure_last(ps_context_t* ctx, double* median_base, double* median_mlp,
                                 int* used, int* samples);

/* after a tick in mode >= 1: the network inputs x (k x 16) and the output
 * scale m s / 100 (k) of the sorted particles idx[0..k) (host arrays) */
ps_result_t ps_b200_closure_features(ps_context_t* ctx, const uint32_t* idx, size_t k,
                                     float* x_out, float* scale_out);

/* after a tick in mode 2: every particle's correction (n x 3, sorted order,
 * host array), whether or not the judge applied it */
ps_result_t ps_b200_closure_correction(ps_context_t* ctx, float* out, size_t n);

/* the network on given inputs (host arrays): y (n x 8) = MLP(x (n x 16)) */
ps_result_t ps_b200_closure_forward(ps_context_t* ctx, const float* x, size_t n,
                                    const float* params, float* y_out);

/* training on the GPU with the project's own kernels: the mean squared error
 * over outputs 0..2 of MLP(x) against t (n x 3) and its gradient for one
 * batch (grad), or Adam over `epochs` shuffled passes of `batch` samples,
 * the learning rate decaying from lr along a cosine to 5 % of it (params in:
 * initial values, out: trained; loss_out: per-epoch MSE) */
ps_result_t ps_b200_closure_grad(ps_context_t* ctx, const float* x, const float* t, size_t n,
                                 const float* params, float* grad_out, float* loss_out);
ps_result_t ps_b200_closure_train(ps_context_t* ctx, const float* x, const float* t, size_t n,
                                  float* params, uint32_t epochs, uint32_t batch, float lr,
                                  uint64_t seed, float* loss_out);

/* ---- batched ensemble (no counterpart in the reference) ----------------
 *
 * Many independent systems advanced together: every phase of a tick -- ids
 * reset, prepare, sort, tree build, upward pass, traversal, velocity
 * permutation + semi-implicit Euler as in ps_b200_run_ticks -- is one launch
 * over all systems (each system sorted and built within its own range, each
 * traversal group with its own system's theta and root), and one tick is two
 * CUDA graphs captured once and replayed.  The systems' particles are one
 * concatenated set of DEVICE arrays: system k holds counts[k] particles from
 * the sum of the counts before it, its ids are local (0 .. counts[k]-1) and,
 * like its positions, come back sorted within its range.  Results equal
 * running each system through ps_b200_run_ticks with its own theta and leaf
 * capacity, bit for bit.  At most 65,536 systems. */
typedef struct ps_b200_ensemble ps_b200_ensemble_t;

/* theta per system (NULL: 2.0 for all) */
ps_result_t ps_b200_ensemble_create(ps_b200_ensemble_t** out, const size_t* counts,
                                    size_t n_systems, const float* theta);

/* The autotuner, on copies of the given state (arrs and the codes array are
 * not changed): per expansion order it may try (ps_b200_ensemble_set_order;
 * default both), per leaf capacity of the ladder (default {1, 16, 32, 64})
 * and size class (systems with equal floor(log2 N)), the smallest theta of
 * {1, 1.5, 2, 3, 4, 6, 8} whose median relative force error against an FP64
 * direct sum (1024 sampled particles of the class's first system, ticked
 * alone) is at most target_median_error (none: 8); then, class by class from
 * the one holding the most particles, the leaf capacity (with its theta)
 * whose forces replay of the whole ensemble is fastest among those that met
 * the target, and the order whose result replays fastest; then the
 * traversal grids' scale among {1, 1/2, 1/4}, by the same replay time.
 * theta_out (n_systems) and grid_scale_out receive the
 * choice (either may be NULL); ps_b200_ensemble_leaf_caps reads the leaf
 * capacities. */
ps_result_t ps_b200_ensemble_autotune(ps_b200_ensemble_t* ens, const ps_particle_arrs_t* arrs,
                                      uint32_t* morton_codes, float target_median_error,
                                      float* theta_out, double* grid_scale_out);

/* `ticks` ensemble ticks; vx, vy, vz are concatenated device arrays too */
ps_result_t ps_b200_ensemble_run(ps_b200_ensemble_t* ens, const ps_particle_arrs_t* arrs,
                                 uint32_t* morton_codes, float* vx, float* vy, float* vz,
                                 float dt, uint32_t ticks);
ps_result_t ps_b200_ensemble_theta(ps_b200_ensemble_t* ens, float* theta_out, size_t n);
/* leaf capacity (PS_B200_OPT_LEAF_CAP) of each system: read, set (n = n_systems) */
ps_result_t ps_b200_ensemble_leaf_caps(ps_b200_ensemble_t* ens, uint32_t* cap_out, size_t n);
ps_result_t ps_b200_ensemble_set_leaf_caps(ps_b200_ensemble_t* ens, const uint32_t* caps,
                                           size_t n);
/* the leaf capacities the autotuner tries (each 1..256) */
ps_result_t ps_b200_ensemble_set_leaf_ladder(ps_b200_ensemble_t* ens, const uint32_t* caps,
                                             size_t n);
/* local expansion of all systems: 0 the reference's (default), 1 the order-1
 * expansion of the closure's mode 1 (PS_B200_OPT_CLOSURE); a negative order
 * lets ps_b200_ensemble_autotune try both and keep the faster at its target
 * error, which ps_b200_ensemble_order then reads back */
ps_result_t ps_b200_ensemble_set_order(ps_b200_ensemble_t* ens, int order);
ps_result_t ps_b200_ensemble_order(ps_b200_ensemble_t* ens, int* order_out);
ps_result_t ps_b200_ensemble_destroy(ps_b200_ensemble_t* ens);

/* message of the last CUDA-side failure on this thread */
const char* ps_b200_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* POLESITTER_B200_H */
