/*
 * fa2b200.h -- C ABI of the B200 ForceAtlas2 engine (libfa2b200.so).
 *
 * This is the boundary under the reference's C++ interface: the drop-in
 * RPGraph::CUDAForceAtlas2 (include/RPGPUForceAtlas2.hpp) is a thin shim over
 * these calls, and any FFI (ctypes, cgo, JNI) can bind them directly.  Plain
 * C types only: no CUDA or torch types cross this boundary.
 *
 * Conventions
 *  - Node ids are the reference's: 0..num_nodes-1 as UGraph assigns them
 *    (first appearance in the edge list).  Position and force arrays are
 *    interleaved x,y pairs in that id order.
 *  - Every call returns a status (FA2_OK = 0) instead of exiting, which is
 *    what the reference does on a CUDA error (src/RPCommon.hpp:33-41); the
 *    C++ shim turns a nonzero status back into that print-and-exit.
 *  - All state lives in the context; any number of contexts may coexist
 *    (the reference keeps its speed and tree state in device statics,
 *    src/RPFA2Kernels.cu:29-33 and src/RPBHKernels.cu:58-62, so it allows one).
 *  - Calls on one context are not thread-safe; use one host thread per context.
 */
#ifndef FA2B200_H
#define FA2B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum fa2_status {
    FA2_OK = 0,
    FA2_ERR_INVALID_ARGUMENT = 1, /* bad pointer, size, id, or a self-loop */
    FA2_ERR_NO_DEVICE = 2,        /* no CUDA device, or not an sm_100 part */
    FA2_ERR_CUDA = 3,             /* a CUDA runtime call failed */
    FA2_ERR_OUT_OF_MEMORY = 4,
    FA2_ERR_DEVICE_LIMIT = 5,     /* a device-side bound was hit (see fa2_get_stats) */
    FA2_ERR_TOO_LARGE = 6,        /* graph beyond the engine's index ranges */
    FA2_ERR_UNSUPPORTED = 7,      /* e.g. exact (non-Barnes-Hut) repulsion */
    FA2_ERR_IO = 8                /* a file could not be read or written */
};

typedef struct fa2_ctx fa2_ctx;

/* An undirected graph: each edge once, no self-loops, ids < num_nodes.
 * Replaces the graph half of the CUDAForceAtlas2 constructor
 * (src/RPGPUForceAtlas2.cu:51-84), which reads UGraph::neighbors_with_geq_id.
 * weights (may be NULL) gives each edge a weight w > 0, in the order of
 * sources/targets; with fa2_params.delta != 0 an edge attracts with
 * w^delta times the unweighted force.  UGraph has no weights and the
 * reference's GPU path no edge weight influence (ForceAtlas2::delta,
 * src/RPForceAtlas2.hpp:49, is 0 and unread), so the drop-in passes NULL. */
typedef struct {
    uint32_t num_nodes;
    uint64_t num_edges;
    const uint32_t *sources;
    const uint32_t *targets;
    const float *weights;
} fa2_graph_desc;

/* The ForceAtlas2 parameters of src/RPForceAtlas2.cpp:28-55. */
typedef struct {
    int32_t use_barneshut;    /* must be 1: the GPU path is Barnes-Hut only
                                 (src/graph_viewer.cpp:93-97) */
    int32_t strong_gravity;   /* 1: f_g = k_g m; 0: f_g = k_g m / |p| */
    float gravity;            /* k_g (setGravity) */
    float scale;              /* k_r (setScale) */
    float theta;              /* Barnes-Hut accuracy, 1.0 (:45) */
    float epssq;              /* softening, 0.05^2 (:46) */
    float jitter_tolerance;   /* 1.0 (:40) */
    float k_s_max;            /* 10.0 (:43) */
    int32_t device;           /* CUDA device ordinal */
    int32_t linlog;           /* 1: linear-log attraction, f_a = log(1 + d) (use_linlog,
                                 src/RPForceAtlas2.hpp:44; honoured by the reference's
                                 CPU path only, src/RPCPUForceAtlas2.cpp:59-67).  0 by
                                 default, as in the reference (src/RPForceAtlas2.cpp:52) */
    int32_t multipole;        /* 1 (default): cells act as point masses at their centre
                                 of mass, as in the reference (src/RPBHKernels.cu:661-668);
                                 2: each accepted cell also adds its quadrupole term (no
                                 reference counterpart; see fa2_set_approximation) */
    float delta;              /* edge weight influence (ForceAtlas2::delta,
                                 src/RPForceAtlas2.hpp:49; 0 by default, :49 of
                                 src/RPForceAtlas2.cpp): the attraction of an edge of
                                 weight w is w^delta times the unweighted one, linear or
                                 linear-log.  Used only with fa2_graph_desc.weights; 0
                                 ignores the weights.  No counterpart on the reference's
                                 GPU path. */
} fa2_params;

/* Fills the reference defaults (weak gravity, gravity 1, scale 1). */
void fa2_default_params(fa2_params *p);

/* Replaces the CUDAForceAtlas2 constructor (src/RPGPUForceAtlas2.cu:37-162):
 * builds the device graph and all per-iteration buffers.  Positions start at
 * zero; call fa2_set_positions.  Returns NULL and sets *status on failure. */
fa2_ctx *fa2_create(const fa2_graph_desc *graph, const fa2_params *params, int *status);

/* Replaces ~CUDAForceAtlas2 (src/RPGPUForceAtlas2.cu:192-204). */
void fa2_destroy(fa2_ctx *ctx);

/* Replaces sendLayoutToGPU (src/RPGPUForceAtlas2.cu:256-260): xy holds
 * 2*num_nodes floats (host memory; pinned memory makes the copy faster).
 * Like the reference it copies positions only; previous forces and the
 * adaptive speed are kept (fa2_set_speed_state resets them). */
int fa2_set_positions(fa2_ctx *ctx, const float *xy);

/* Replaces retrieveLayoutFromGPU (src/RPGPUForceAtlas2.cu:250-254), the data
 * half of sync_layout (:270-278). */
int fa2_get_positions(fa2_ctx *ctx, float *xy);

/* Replaces CUDAForceAtlas2::doStep (src/RPGPUForceAtlas2.cu:206-248), run
 * n_iters times; returns when the device has finished, like doStep's
 * cudaDeviceSynchronize (:246). */
int fa2_step(fa2_ctx *ctx, int32_t n_iters);

/* fa2_set_positions(xy_in), fa2_step(n_iters) and fa2_get_positions(xy_out)
 * in one call, with one synchronisation of the host instead of three: the
 * copies, the iterations and the state read that follows them are queued
 * together.  xy_in and xy_out (2 floats per node, reference order) may each
 * be NULL, and may be the same buffer; from pinned memory the copies run at
 * the link's rate.  The positions and forces are those of the three calls,
 * bit for bit.  An iteration that must be replayed (coincident bodies) and
 * an active accuracy guard take the path of the three calls.  No reference
 * counterpart: a host loop that owns the positions (graph_viewer writes
 * them out between runs of iterations) calls this once per round trip. */
int fa2_step_host(fa2_ctx *ctx, const float *xy_in, int32_t n_iters, float *xy_out);

/* fa2_step with device timing: *ms_total receives the CUDA-event time of
 * the whole call on the engine's stream.  With kernel_ms (n_kernels > 0) the
 * iterations run a copy of the iteration graph with an event before and
 * after each kernel, and kernel_ms receives, for each kernel listed by
 * fa2_kernel_name, its mean duration per launch in ms over the call; those
 * events cost time of their own, most on small graphs.  With kernel_ms NULL
 * (or n_kernels 0) the iterations run fa2_step's graph, with events only
 * around the call.  No reference counterpart: it serves measurement. */
int fa2_step_timed(fa2_ctx *ctx, int32_t n_iters, float *ms_total, float *kernel_ms,
                   int32_t n_kernels);

/* Name of timed kernel slot i, or NULL past the last one. */
const char *fa2_kernel_name(int32_t i);

/* Diagnostics of the last step; test and measurement hooks with no
 * reference counterpart. */
typedef struct {
    uint32_t num_bodies;
    uint32_t tree_nodes;        /* cells + bodies of the last quadtree */
    uint32_t tree_cells;
    int32_t max_level;          /* deepest cell level (root 0) */
    int32_t perturb_rounds;     /* .99 re-insertion rounds in the last step */
    int32_t device_error;       /* bit set of device-side limit hits, 0 = none:
                                   2 tree-count wait limit, 4 more than 1024 bodies on
                                   one 64-bit key, 8 tree larger than its buffer,
                                   16 a NaN or infinite position.  Stepping stops
                                   while one is set; fa2_set_positions clears them */
    uint64_t nnz_padded;        /* CSR entries incl. padding */
    float global_speed;         /* adaptive speed after the last step */
    float speed_efficiency;
    float radius, root_x, root_y;
    uint64_t interactions;      /* body-node force terms of the last traversal */
    uint64_t visits;            /* body-node acceptance tests of the last traversal */
    int32_t sort_passes;        /* 8-bit digit passes of the last step's sorts: 8; 6
                                   after a tree no deeper than level 22, 7 after one no
                                   deeper than 26 (runs of keys equal in the sorted
                                   top bits are then ordered by a fix-up pass) */
    uint64_t learned_pairs;     /* (group, cell) pairs the last learned iteration's walk
                                   collected for the MLP (0 without the learned
                                   correction; see fa2_set_learned_correction) */
} fa2_stats;

int fa2_get_stats(fa2_ctx *ctx, fa2_stats *out);

/* Last step's forces before displacement (test hook): f_total is the full
 * FA2 force, f_attr_grav the gravity + attraction part; either may be NULL.
 * The reference keeps these in fxl/fyl (src/RPGPUForceAtlas2.cu:136-139). */
int fa2_get_forces(fa2_ctx *ctx, float *f_total, float *f_attr_grav);

/* Last step's body order of the quadtree, as node ids: the reference's sortd
 * (src/RPBHKernels.cu:513-559). */
int fa2_get_sort_order(fa2_ctx *ctx, uint32_t *order);

/* Overwrites the adaptive speed state (global_speed, speed_efficiency) and the
 * previous forces (2*num_nodes floats, or NULL for zero).  Checkpoint/restore
 * hook: the reference never saves these (src/RPGraphLayout.cpp:228-250). */
int fa2_set_speed_state(fa2_ctx *ctx, float global_speed, float speed_efficiency,
                        const float *f_prev);
int fa2_get_speed_state(fa2_ctx *ctx, float *global_speed, float *speed_efficiency,
                        float *f_prev);

/* Changes k_r and k_g between steps: ForceAtlas2::setScale / setGravity
 * (src/RPForceAtlas2.cpp:64-72), which the reference passes to every launch. */
int fa2_set_force_params(fa2_ctx *ctx, float scale, float gravity);

/* Switches between linear (0) and linear-log (1) attraction between steps:
 * fa2_params.linlog after creation.  No counterpart on the reference's GPU
 * path, which ignores ForceAtlas2::use_linlog. */
int fa2_set_linlog(fa2_ctx *ctx, int32_t enable);

/* Far-field accuracy between steps, no reference counterpart (its theta is
 * fixed at 1, src/RPForceAtlas2.cpp:45).  theta > 0 is the Barnes-Hut opening
 * parameter (the acceptance test d^2 + eps >= (2 r)^2 / theta^2 + eps);
 * multipole 1 uses each accepted cell as a point mass, as the reference does;
 * multipole 2 adds the cell's quadrupole term conj(a2 / w^3), a2 = sum m (z - Z)^2
 * over the cell's bodies about its centre of mass Z, w = p_i - Z with the
 * softened |w|^2 = d^2 + eps.  The quadrupole at a larger theta reaches the
 * monopole's error at theta = 1 with fewer node visits.  FA2_ERR_INVALID_ARGUMENT
 * for theta <= 0 or multipole outside 1..2. */
int fa2_set_approximation(fa2_ctx *ctx, float theta, int32_t multipole);

/* Exact all-pairs repulsion of sampled nodes, in double precision on the GPU,
 * at the current positions: out[2 s], out[2 s + 1] = k_r m_i sum_{j != i} m_j d /
 * (d^2 + eps) for i = samples[s] (reference ids), d = p_i - p_j.  The yardstick
 * for the tree's approximation error; no reference counterpart. */
int fa2_exact_repulsion(fa2_ctx *ctx, int32_t n_samples, const uint32_t *samples, double *out);

/* Accuracy guard for an approximation other than the reference's (theta != 1
 * or multipole 2); no reference counterpart.  Every `every` iterations of
 * fa2_step / fa2_step_timed, after that iteration, the repulsion it applied to
 * n_samples bodies spread evenly over the sorted order is compared with the
 * exact FP64 sum over all bodies, and so is the reference walk (monopole,
 * theta 1) over the same tree.  If the applied repulsion has the larger
 * relative RMSE, the context falls back to the reference walk for the
 * iterations that follow (fa2_set_approximation selects an approximation
 * again).  every = 0 turns the guard off.  A check costs one FP64 sum over all
 * bodies per sample.  Resets the counts of fa2_get_accuracy_guard. */
int fa2_set_accuracy_guard(fa2_ctx *ctx, int32_t every, int32_t n_samples);

/* The last check's relative RMSE of the applied and of the reference walk's
 * repulsion against the FP64 sum, and the numbers of checks and of fallbacks
 * since fa2_set_accuracy_guard.  Null pointers are skipped. */
int fa2_get_accuracy_guard(fa2_ctx *ctx, double *err_current, double *err_plain,
                           int32_t *checks, int32_t *fallbacks);

/* The last CUDA error a call of this thread met that returned FA2_ERR_CUDA or
 * FA2_ERR_OUT_OF_MEMORY: its name, text and the source line that saw it; ""
 * if none.  The string stays valid until this thread's next failing call. */
const char *fa2_last_cuda_error(void);

/* ------------------------------------------------------------------------
 * Learned far-field correction.  No counterpart in the reference: its walk
 * adds every accepted cell as a point mass at its centre of mass
 * (src/RPBHKernels.cu:656-668), and that term is what the correction mends.
 *
 * A warp walks the tree for a group of 32 sorted bodies and accepts a cell
 * only if all 32 pass the cell test.  Every (group, accepted cell) pair goes
 * through a 12 -> 64 -> 64 -> 2 MLP.  Its features are the cell's multipole
 * statistics as the group sees them: mass, second moments, width, level and
 * acceptance margin, plus the group's spread and moments, taken relative to
 * the distance d from the cell's centre of mass to the group's centroid, in a
 * frame turned to that direction.  Its two outputs, turned back and
 * multiplied by M / d, estimate the mean over the group's bodies of the error
 * the walk's term makes for that cell.  Each body of the group receives k_r
 * m_i times the sum of its pairs' estimates.
 * The MLP runs on the tensor cores with BF16 weights and activations and
 * FP32 accumulation.  A pair whose group spread is more than half of d gets
 * no correction.
 * ---------------------------------------------------------------------- */

#define FA2_MLP_IN 12
#define FA2_MLP_HIDDEN 64
#define FA2_MLP_OUT 2

/* The MLP's parameters in FP32, laid out like PyTorch's nn.Linear weights
 * ([out][in], row-major).  Inference rounds w1, w2 and w3 and the hidden
 * activations to BF16; the biases stay FP32. */
typedef struct fa2_mlp {
    float w1[FA2_MLP_HIDDEN * FA2_MLP_IN];
    float b1[FA2_MLP_HIDDEN];
    float w2[FA2_MLP_HIDDEN * FA2_MLP_HIDDEN];
    float b2[FA2_MLP_HIDDEN];
    float w3[FA2_MLP_OUT * FA2_MLP_HIDDEN];
    float b3[FA2_MLP_OUT];
} fa2_mlp;

/* PyTorch's default initialisation of nn.Linear: every weight and bias
 * uniform in +-1/sqrt(fan_in), drawn from a generator seeded with seed. */
void fa2_mlp_init(fa2_mlp *mlp, uint32_t seed);

/* Turns the correction on for the iterations that follow (mlp != NULL), on
 * top of the walk fa2_set_approximation selected (theta, multipole 1 or 2);
 * NULL turns it off.  The weights are copied.  A learned iteration also runs
 * the moment scan of the quadrupole option (the features need each cell's
 * second moment), the MLP and a separate tail kernel for the force sum and
 * the speed rule.  With all-zero weights it gives the plain walk's forces
 * and positions bit for bit.  The accuracy guard (fa2_set_accuracy_guard)
 * checks the corrected repulsion and, on a fallback, also turns the
 * correction off. */
int fa2_set_learned_correction(fa2_ctx *ctx, const fa2_mlp *mlp);

/* Launch shape of the MLP kernel on `device`: thread blocks per SM (each a
 * 128-row tile loop holding 64 tensor-memory columns) and dynamic shared
 * memory per block. */
int fa2_mlp_launch_shape(int32_t device, int32_t *blocks_per_sm, int32_t *smem_bytes);

/* The inference kernel alone: out[2 r], out[2 r + 1] = MLP(features[12 r ..
 * 12 r + 11]) for n rows (host arrays), on CUDA device `device`. */
int fa2_mlp_forward(int32_t device, const fa2_mlp *mlp, const float *features, int64_t n,
                    float *out);

/* The training kernels alone: one Adam step (PyTorch's Adam with its default
 * betas 0.9, 0.999 and eps 1e-8; `step` counts from 1) over n samples (host
 * arrays: features n x 12, targets n x 2, weights n) of the loss
 * sum_s min(w_s, 100) |MLP(x_s) - t_s|^2 / (2 n), in FP32.  params, adam_m and
 * adam_v are updated in place; *loss (if not NULL) receives the loss before
 * the step. */
int fa2_mlp_train_step(int32_t device, fa2_mlp *params, fa2_mlp *adam_m, fa2_mlp *adam_v,
                       int32_t step, float lr, const float *features, const float *targets,
                       const float *weights, int32_t n, float *loss);

/* Training samples held in device memory. */
typedef struct fa2_learn_set fa2_learn_set;

/* Room for `capacity` samples on CUDA device `device` (60 bytes each). */
fa2_learn_set *fa2_learn_set_create(int32_t device, int64_t capacity, int *status);
void fa2_learn_set_destroy(fa2_learn_set *set);
int64_t fa2_learn_set_size(const fa2_learn_set *set);

/* Adds the samples of ctx's current positions: builds the tree, walks it at
 * `theta` with `multipole` (the walk the correction will be used on) and, for
 * every (group, cell) pair that passes the spread test, stores its features,
 * its target (the exact FP64 mean over the group's bodies of the error of the
 * walk's term for that cell, turned and scaled as the MLP's outputs are) and
 * its weight ((M/d)^2 times the sum of the group's squared masses: the
 * pair's share of the squared force error).  The samples of one call are
 * stored in (group, node) order.  Positions, speeds and the forces of the
 * last step are left as they were; the tree, sort order and fa2_get_stats
 * then describe this walk.  Samples past the capacity are dropped (*added
 * counts those stored).  Coincident bodies stop the walk: nothing is added. */
int fa2_learn_collect(fa2_learn_set *set, fa2_ctx *ctx, float theta, int32_t multipole,
                      int64_t *added);

/* Copies samples [first, first + count) to host arrays (NULL skips one). */
int fa2_learn_set_read(const fa2_learn_set *set, int64_t first, int64_t count, float *features,
                       float *targets, float *weights);

/* Trains mlp (in place, from its current values) for `steps` Adam steps on
 * batches of `batch` samples: the set in a random order drawn from `seed`,
 * reshuffled at every pass; weights scaled to a mean of 1 over the set;
 * learning rate lr decaying exponentially to lr / 20 at the last step.
 * *final_loss (if not NULL) is the last batch's loss. */
int fa2_learn_fit(fa2_learn_set *set, fa2_mlp *mlp, int32_t steps, int32_t batch, float lr,
                  uint32_t seed, float *final_loss);

/* prevent_overlap (ForceAtlas2::prevent_overlap, src/RPForceAtlas2.hpp:44),
 * which the reference declares but never implements: its CPU displacement
 * exits with "Not yet implemented" (src/RPCPUForceAtlas2.cpp:201-205) and its
 * GPU path does not read the flag.  Here it is the rule of the ForceAtlas2
 * paper (Jacomy et al., PLoS ONE 2014) on the border-to-border distance
 * d' = d - s_i - s_j between bodies of sizes s (reference id order, one per
 * node, finite and >= 0): repulsion k_r m_i m_j / d' while apart, 100 k_r
 * m_i m_j while overlapping, nothing at d' = 0; attraction d' while apart,
 * nothing while overlapping (times w^delta with edge weights).  d is the
 * walk's softened distance sqrt(d^2 + eps) in the repulsion.  A Barnes-Hut
 * cell has no size and repels as a point mass.  With every size 0 the forces
 * are those of the plain rule up to float rounding (the overlap form goes
 * through a square root).  NULL turns it off.  FA2_ERR_UNSUPPORTED with linear-log attraction,
 * the quadrupole walk, the learned correction or the accuracy guard. */
int fa2_set_prevent_overlap(fa2_ctx *ctx, const float *sizes);

/* Measurement hook, no reference counterpart.  enable = 1 (the default) runs
 * the attraction on a second stream beside the tree build, the two sharing
 * the GPU; enable = 0 runs it alone before the tree build, so that the
 * per-kernel times of fa2_step_timed are those of each kernel on its own.
 * Results are the same either way. */
int fa2_set_overlap(fa2_ctx *ctx, int32_t enable);

/* ------------------------------------------------------------------------
 * Batched layout: many independent graphs in one persistent launch.  No
 * counterpart in the reference, which lays out one graph per process (its
 * speed and tree state are device statics, src/RPFA2Kernels.cu:29-33,
 * src/RPBHKernels.cu:54-62).  Every graph gets the FA2 iteration of
 * fa2_step with its own quadtree, speed state and bounding box; one CTA runs
 * a graph's iterations, taking graphs largest first from a queue.
 * ---------------------------------------------------------------------- */

typedef struct fa2_batch fa2_batch;

/* Largest graph (nodes) the batched path takes; larger ones -> FA2_ERR_TOO_LARGE. */
#define FA2_BATCH_MAX_NODES 65536

/* num_graphs graphs, each as fa2_create takes one (ids local to the graph);
 * the parameters apply to every graph.  Positions start at zero. */
/* params->multipole must be 1, and edge weights need params->delta == 0
 * (FA2_ERR_UNSUPPORTED otherwise). */
fa2_batch *fa2_batch_create(uint32_t num_graphs, const fa2_graph_desc *graphs,
                            const fa2_params *params, int *status);
void fa2_batch_destroy(fa2_batch *batch);

/* Positions of all graphs, graph after graph, each graph's nodes in id order
 * (2 floats per node; host memory). */
int fa2_batch_set_positions(fa2_batch *batch, const float *xy);
int fa2_batch_get_positions(fa2_batch *batch, float *xy);

/* n_iters iterations of every graph in one launch; returns when done.
 * FA2_ERR_DEVICE_LIMIT if a graph hit a device bound (its iterations stop). */
int fa2_batch_step(fa2_batch *batch, int32_t n_iters);

/* fa2_batch_step with *ms = CUDA-event time of the launch. */
int fa2_batch_step_timed(fa2_batch *batch, int32_t n_iters, float *ms);

/* Test hooks, last iteration: total and gravity + attraction forces (2 floats
 * per node, same order as the positions); the body order of each graph's
 * quadtree (graph-local ids, the reference's sortd); the adaptive speed and
 * speed efficiency per graph. */
/* CTA sizes: graphs of at most `split` nodes run on CTAs of small_threads
 * threads beside the others on CTAs of large_threads threads (each 256, 512
 * or 1024), each class from its own queue; the default is split 0 with
 * 1024-thread CTAs, one class.  Results do not depend on the choice, only the
 * speed does. */
int fa2_batch_configure(fa2_batch *batch, uint32_t split, int32_t small_threads,
                        int32_t large_threads);
int fa2_batch_get_config(fa2_batch *batch, uint32_t *split, int32_t *small_threads,
                         int32_t *large_threads);

/* Picks the configuration by measurement: times `iters` iterations of every
 * candidate on this batch (large CTAs of 1024 or 512 threads; no split, or
 * graphs up to 256, 1024 or 4096 nodes on CTAs of 256 or 512 threads; or all
 * graphs on the small CTAs), keeps the fastest, and puts the layout state
 * (positions, speeds, and the forces and orders of the last iteration) back
 * as it was.  Returns the choice and its ms per iteration. */
int fa2_batch_autotune(fa2_batch *batch, int32_t iters, uint32_t *split,
                       int32_t *small_threads, int32_t *large_threads, float *ms_per_iter);

int fa2_batch_get_forces(fa2_batch *batch, float *f_total, float *f_attr_grav);
int fa2_batch_get_sort_order(fa2_batch *batch, uint32_t *order);
int fa2_batch_get_speed(fa2_batch *batch, float *global_speed, float *speed_efficiency);

/* ------------------------------------------------------------------------
 * Repulsion without allocation.  No counterpart in the reference: there the
 * repulsion runs only inside CUDAForceAtlas2::doStep, on buffers that the
 * constructor allocated (src/RPGPUForceAtlas2.cu:109-149).
 * ---------------------------------------------------------------------- */

/* Largest body count fa2_repulsion_noalloc accepts. */
#define FA2_NOALLOC_MAX_BODIES 8192

/* Barnes-Hut repulsion of n bodies whose positions (d_xy, n interleaved x,y
 * floats) and masses (d_mass) already sit in device memory of prm->device;
 * writes the n repulsive forces (interleaved x,y) to d_force there.  They are
 * the repulsion fa2_step computes for the same positions and masses: the same
 * quadtree, cell test (prm->theta, prm->epssq) and strength k_r = prm->scale.
 * Gravity, attraction, the speed rule and the displacement are not applied.
 *
 * For callers that must not allocate at the point of the call: code under a
 * fixed device-memory budget, or inside a host framework whose caching
 * allocator it may not touch, or a process that reserved the device's memory
 * up front.  No call allocates device or host memory.  All scratch lives in
 * one fixed array in the library's device memory, about 6 MB per device,
 * held from the time the library's kernels are loaded on that device.
 *
 *  - n > FA2_NOALLOC_MAX_BODIES returns FA2_ERR_TOO_LARGE before any work.
 *  - The first call on a device does set-up: it looks up the scratch array's
 *    address with that device current and sets kernel attributes (and, like
 *    any first CUDA call, may create the device's context).  Make it before
 *    any stream capture.
 *  - The work is enqueued on `stream` (a cudaStream_t; NULL is the default
 *    stream); the call then copies two device flags to host memory and
 *    waits for that stream (cudaStreamSynchronize) before it returns, and
 *    reports: coincident bodies, a NaN or infinite position, or a mass that
 *    is not a whole number in [0, 2^24) -> FA2_ERR_INVALID_ARGUMENT (fa2_step moves coincident bodies
 *    apart, and its masses are degree + 1; this call does neither), a
 *    device-side bound -> FA2_ERR_DEVICE_LIMIT.
 *  - There is one scratch array per device: calls that overlap on the same
 *    device (several host threads, or several streams) race on it and give
 *    wrong forces.  Serialise them.
 *  - d_xy and d_force 8-byte aligned, d_mass 4-byte aligned; d_force must not
 *    overlap d_xy or d_mass.
 *  - prm->multipole must be 1: 2 (the quadrupole walk) gives
 *    FA2_ERR_UNSUPPORTED, a value below 1 FA2_ERR_INVALID_ARGUMENT.
 *  - Launch errors are read from the CUDA runtime's last-error slot only when
 *    that slot was empty on entry: an error the caller left there is neither
 *    reported as this call's nor cleared. */
int fa2_repulsion_noalloc(const float *d_xy, const float *d_mass, uint32_t n,
                          const fa2_params *prm, void *stream, float *d_force);

/* ------------------------------------------------------------------------
 * Host graph layer: RPGraph::UGraph and GraphLayout behind plain C, for
 * callers that bind the C ABI instead of the C++ classes.
 * ---------------------------------------------------------------------- */

typedef struct fa2_ugraph fa2_ugraph;

/* RPGraph::UGraph::UGraph(path) (src/RPGraph.cpp:35-56): ids by first
 * appearance, self-loops and repeated undirected edges dropped.  NULL with
 * FA2_ERR_IO when the file cannot be opened. */
fa2_ugraph *fa2_ugraph_load(const char *path, int *status);

/* The same from n_pairs (s, t) pairs already in memory, in file order. */
fa2_ugraph *fa2_ugraph_from_pairs(const uint32_t *s, const uint32_t *t, uint64_t n_pairs,
                                  int *status);
void fa2_ugraph_free(fa2_ugraph *g);
uint32_t fa2_ugraph_num_nodes(const fa2_ugraph *g);
uint64_t fa2_ugraph_num_edges(const fa2_ugraph *g);

/* node_map_r: UGraph id -> edge-list id (num_nodes entries). */
int fa2_ugraph_node_map_r(const fa2_ugraph *g, uint32_t *out);

/* UGraph::degree of every node (num_nodes entries). */
int fa2_ugraph_degrees(const fa2_ugraph *g, uint32_t *out);

/* All edges as CUDAForceAtlas2 lists them (src/RPGPUForceAtlas2.cu:77-84):
 * sources ascending, each source's neighbors_with_geq_id in order. */
int fa2_ugraph_edges(const fa2_ugraph *g, uint32_t *sources, uint32_t *targets);

/* srandom(seed), then GraphLayout(graph, width, height).randomizePositions()
 * (src/RPGraphLayout.cpp:45-52): 2*n floats, x then y per node. */
void fa2_random_positions(uint32_t n, float width, float height, uint32_t seed, float *xy);

/* GraphLayout::writeToCSV / writeToBin (src/RPGraphLayout.cpp:209-250) of
 * positions xy for graph g.  Refuses (FA2_ERR_IO) an existing file. */
int fa2_write_layout(const fa2_ugraph *g, const float *xy, const char *path, int binary);

/* ------------------------------------------------------------------------
 * Headless rendering: the picture of GraphLayout::writeToPNG
 * (src/RPGraphLayout.cpp:170-207) drawn on the GPU.  Every node is a filled
 * disc of radius 3 px blended black at opacity 10000 / num_nodes, every edge
 * a line blended black at opacity 100000 / num_edges, on white, the layout's
 * bounding box scaled to the image.  Blending black scales a pixel by
 * (1 - opacity), so the image is a product over the plots covering each
 * pixel, independent of drawing order.  pngwriter, which the reference draws
 * with, is not part of its sources; the pixel rules are: positions truncated
 * to int as the reference computes them, pixel (x, y) 1-based with y up; a
 * disc is every pixel within distance 3; a line the Bresenham pixels between
 * its integer end points.
 * ---------------------------------------------------------------------- */

/* Renders into rgb (image_w * image_h * 3 bytes, top row first) on CUDA device
 * `device`.  Edges as fa2_ugraph_edges lists them, each once. */
int fa2_render_rgb(uint32_t num_nodes, uint64_t num_edges, const uint32_t *sources,
                   const uint32_t *targets, const float *xy, int32_t image_w, int32_t image_h,
                   int32_t device, uint8_t *rgb);

/* Writes an 8-bit RGB PNG of rgb (image_w * image_h * 3 bytes, top row first). */
int fa2_png_encode(const uint8_t *rgb, int32_t image_w, int32_t image_h, const char *path);

/* GraphLayout::writeToPNG of positions xy for graph g, rendered on device 0;
 * like the reference it overwrites an existing file. */
int fa2_write_png(const fa2_ugraph *g, const float *xy, int32_t image_w, int32_t image_h,
                  const char *path);

/* Human-readable text of a status code. */
const char *fa2_status_string(int status);

/* Library version string. */
const char *fa2_version(void);

#ifdef __cplusplus
}
#endif
#endif
