/*
 * fa2_oracle.h -- CPU restatement of the ForceAtlas2 GPU path of govertb/GPUGraphLayout.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA engine in
 * gpugraphlayout_b200/.  Only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline / reference legs load it, and only to check or to time the CPU
 * baseline.  The engine never links, loads or calls it and has no CPU fallback.
 *
 * Every function restates one piece of the reference, cited as file:line
 * relative to the reference project root.  Floating-point expressions keep the
 * reference's operand order and types (float vs double literals) so that, built
 * without FMA contraction, the results match the reference's own kernels run
 * through the CPU SIMT emulator in oracle/ref (the pin), bit for bit.
 */
#ifndef FA2_ORACLE_H
#define FA2_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- graph -- */

/* RPGraph::UGraph::UGraph (src/RPGraph.cpp:35-56) together with add_node
 * (:79-87) and add_edge (:89-102), applied to an already parsed list of
 * (s, t) pairs in file order: self-loops and repeated undirected edges are
 * dropped, node ids are remapped in first-appearance order (s before t), and
 * every kept edge is recorded as (min, max) of the mapped ids in input order,
 * which is the order of adjacency_list[min].push_back(max).
 * node_map_r needs room for 2*n_pairs entries, e_lo/e_hi for n_pairs.
 * Returns the node count, or -1 when memory runs out. */
int64_t orc_ugraph_build(int64_t n_pairs, const uint32_t *src, const uint32_t *dst,
                         uint32_t *node_map_r, uint32_t *e_lo, uint32_t *e_hi,
                         int64_t *n_edges);

/* The COO edge arrays of CUDAForceAtlas2's constructor
 * (src/RPGPUForceAtlas2.cu:73-84): sources ascending, and for each source its
 * neighbors_with_geq_id in adjacency order; also degree[] (add_edge :99-100). */
void orc_coo_order(int32_t n_nodes, int64_t n_edges, const uint32_t *e_lo,
                   const uint32_t *e_hi, int32_t *sources, int32_t *targets,
                   uint32_t *degree);

/* ------------------------------------------------------------- layout -- */

/* srandom(seed) (src/graph_viewer.cpp:49) followed by
 * GraphLayout::randomizePositions (src/RPGraphLayout.cpp:45-52) with
 * RPGraph::get_random (src/RPCommon.cpp:50-53); xy is interleaved x,y. */
void orc_random_positions(int32_t n, float width, float height, uint32_t seed, float *xy);

/* ------------------------------------------------------- FA2 kernels -- */

/* GravityKernel (src/RPFA2Kernels.cu:35-73); adds to fx, fy. */
void orc_gravity(int32_t n, const float *xy, const float *mass, float k_g,
                 int32_t strong_gravity, float *fx, float *fy);

/* AttractiveForceKernel (src/RPFA2Kernels.cu:75-109) with its atomics applied
 * in edge order; adds to fx, fy. */
void orc_attraction_linlog(int64_t n_edges, const int32_t *sources, const int32_t *targets,
                           const float *xy, float *fx, float *fy);
void orc_attraction(int64_t n_edges, const int32_t *sources, const int32_t *targets,
                    const float *xy, float *fx, float *fy);

/* Edge weight influence (ForceAtlas2::delta, src/RPForceAtlas2.hpp:49): an
 * edge of weight w attracts with w^delta times the force of orc_attraction
 * (linlog 0) or orc_attraction_linlog (linlog 1), the rule F_a = w^delta d of
 * the ForceAtlas2 paper (Jacomy et al., PLoS ONE 9(6), 2014).  wd[e] holds
 * w^delta of edge e.  The reference declares delta but its UGraph has no
 * weights, so nothing of the reference runs this; it restates the published
 * rule in the edge order of the unweighted forms. */
void orc_attraction_weighted(int64_t n_edges, const int32_t *sources, const int32_t *targets,
                             const float *wd, int32_t linlog, const float *xy, float *fx,
                             float *fy);

typedef struct {
    float global_speed;      /* RPFA2Kernels.cu:30, starts at 1 */
    float speed_efficiency;  /* :31, starts at 1 */
    float jitter_tolerance;  /* :32, 1 */
    float k_s_max;           /* :29, 10 */
} orc_speed_state;

void orc_speed_init(orc_speed_state *st);

/* SpeedKernel (src/RPFA2Kernels.cu:111-221).  The swing and traction sums are
 * formed the way one block of `threads` threads forms them (strided partial
 * sums, then the power-of-two tree of :208-217); threads = 512 is the
 * reference's THREADS1.  Updates st and returns the two sums. */
void orc_speed(int32_t n, const float *fx, const float *fy, const float *fxp,
               const float *fyp, const float *mass, int32_t threads,
               orc_speed_state *st, float *swg_sum, float *etra_sum);

/* The global-speed update on given sums (src/RPFA2Kernels.cu:177-219). */
void orc_speed_update(int32_t n, float swg_sum, float etra_sum, orc_speed_state *st);

/* DisplacementKernel (src/RPFA2Kernels.cu:223-251): moves xy, copies f to
 * f_prev and clears f. */
void orc_displacement(int32_t n, float *xy, float *fx, float *fy, float *fxp,
                      float *fyp, float global_speed);

/* ----------------------------------------------------- Barnes-Hut -- */

typedef struct orc_tree orc_tree;

/* BoundingBoxKernel (src/RPBHKernels.cu:70-157) and TreeBuildingKernel
 * (:184-329) run by one thread, so bodies are inserted in id order.  Cell
 * centres follow the kernel's float arithmetic (:217-241) and its tie rule
 * (a coordinate equal to the centre goes to the lower quadrant).  A body that
 * lands exactly on an earlier body is scaled by .99 (a double multiply) and
 * inserted again (:271-278), which changes xy.  Returns NULL when memory runs
 * out.  *n_perturbed counts the .99 scalings. */
orc_tree *orc_tree_build(int32_t n, float *xy, int32_t *n_perturbed);
void orc_tree_free(orc_tree *t);

int32_t orc_tree_maxdepth(const orc_tree *t);   /* maxdepthd (:327-328) */
float orc_tree_radius(const orc_tree *t);       /* radiusd (:140) */
void orc_tree_root(const orc_tree *t, float *cx, float *cy);
int32_t orc_tree_num_cells(const orc_tree *t);

/* SummarizationKernel (src/RPBHKernels.cu:357-506): cell mass, mass-weighted
 * centre of mass and body count, children summed in quadrant order. */
void orc_tree_summarize(orc_tree *t, const float *xy, const float *mass);

/* SortKernel (src/RPBHKernels.cu:513-559): the in-order body permutation
 * sortd[0..n). */
void orc_tree_sort(const orc_tree *t, int32_t *sortd);

/* Per-cell data in depth-first (preorder) order, children in quadrant order:
 * level (root 0), mass, centre of mass, body count.  Arrays hold num_cells. */
void orc_tree_cells(const orc_tree *t, int32_t *level, float *mass, float *cx,
                    float *cy, int32_t *count);

/* ForceCalculationKernel (src/RPBHKernels.cu:566-693): bodies taken in sortd
 * order in groups of `group` (32 is the reference warp); a cell is accepted
 * only if every body of the group passes d^2+eps >= dq[depth], with the
 * per-level dq table of :579-592.  Adds k_r*m_i*m_j*d/(d^2+eps) to fx, fy.
 * Returns 1 and adds nothing when the tree is deeper than 32 levels, as the
 * reference does (:595); 0 otherwise.  n_visits, when not NULL, receives the
 * number of body-node tests summed over bodies. */
int32_t orc_tree_repulsion(const orc_tree *t, const float *xy, const float *mass,
                           float k_r, float itolsq, float epssq, int32_t group,
                           const int32_t *sortd, float *fx, float *fy,
                           int64_t *n_visits);
/* orc_tree_repulsion plus each accepted cell's quadrupole term conj(a2 / w^3)
 * (a2: the cell's complex second moment about its centre of mass; w: the
 * body's offset from it, |w|^2 softened).  No reference counterpart. */
int32_t orc_tree_repulsion_quad(const orc_tree *t, const float *xy, const float *mass,
                                float k_r, float itolsq, float epssq, int32_t group,
                                const int32_t *sortd, float *fx, float *fy, int64_t *n_visits);

/* orc_tree_repulsion with prevent_overlap between bodies (sizes per node):
 * the ForceAtlas2 paper's anti-collision repulsion on the border-to-border
 * distance; cells repel as point masses.  No reference implementation: the
 * reference declares prevent_overlap (RPForceAtlas2.hpp:44) and exits on it
 * (RPCPUForceAtlas2.cpp:201-205). */
int32_t orc_tree_repulsion_overlap(const orc_tree *t, const float *xy, const float *mass,
                                   const float *sizes, float k_r, float itolsq, float epssq,
                                   int32_t group, const int32_t *sortd, float *fx, float *fy,
                                   int64_t *n_visits);

/* Attraction with prevent_overlap: per edge (p_t - p_s) (d - s_s - s_t) / d
 * while the nodes are apart, nothing while they overlap. */
void orc_attraction_overlap(int64_t n_edges, const int32_t *sources, const int32_t *targets,
                            const float *sizes, const float *xy, float *fx, float *fy);

/* Exact pairwise repulsion in double precision for the listed nodes:
 * F_i = sum_{j != i} k_r m_i m_j (p_i - p_j) / (|p_i - p_j|^2 + eps),
 * the force of src/RPCPUForceAtlas2.cpp:92-101 with the GPU softening eps
 * (src/RPBHKernels.cu:651).  Runs one thread per core over the samples. */
void orc_exact_repulsion_f64(int32_t n, const float *xy, const float *mass, double k_r,
                             double eps, int32_t n_samples, const int32_t *samples,
                             double *fx, double *fy);

/* ------------------------------------------------------- full step -- */

typedef struct {
    int32_t n;
    int64_t m;
    const int32_t *sources, *targets;   /* COO edges, orc_coo_order */
    float *xy;                          /* 2n, interleaved */
    const float *mass;                  /* n: degree + 1 */
    float *fx, *fy, *fxp, *fyp;         /* n each */
    float k_r, k_g;
    int32_t strong_gravity;
    float itolsq, epssq;                /* RPForceAtlas2.cpp:45-47 */
    int32_t group;                      /* 32 */
    int32_t speed_threads;              /* 512 */
    orc_speed_state speed;
    /* optional outputs of the last step (may be NULL) */
    int32_t *sortd_out;                 /* n */
    float *f_ga_out;                    /* 2n: gravity + attraction, interleaved */
    float *f_tot_out;                   /* 2n: total force before displacement */
    /* diagnostics: maxdepth is the running maximum over steps (start it at
     * 1, as maxdepthd starts), the others describe the last step */
    int32_t maxdepth, n_perturbed, depth_overflow;
    float swg_sum, etra_sum;
    int32_t linlog;                     /* 1: linear-log attraction */
    const float *sizes;                 /* n node sizes: prevent_overlap; NULL: off */
} orc_fa2;

/* One CUDAForceAtlas2::doStep (src/RPGPUForceAtlas2.cu:206-248) in its kernel
 * order: gravity, attraction, bounding box + tree, summarization, sort,
 * repulsion, speed, displacement.  Returns 0, or -1 when memory runs out. */
int32_t orc_fa2_step(orc_fa2 *s);

#ifdef __cplusplus
}
#endif
#endif
