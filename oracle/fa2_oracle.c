/*
 * fa2_oracle.c -- CPU restatement of the ForceAtlas2 GPU path of
 * govertb/GPUGraphLayout.  TEST INFRASTRUCTURE ONLY: the checker for the CUDA
 * engine, never called by it.  See fa2_oracle.h for the contract and the
 * reference file:line each function restates.
 *
 * Build without FMA contraction (-ffp-contract=off): the expressions below keep
 * the reference's operand order so that results can be compared bit for bit
 * with the reference kernels executed by the CPU emulator in oracle/ref.
 */
#define _DEFAULT_SOURCE
#include "fa2_oracle.h"

#include <float.h>
#include <math.h>
#include <pthread.h>
#include <unistd.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ hash -- */

/* Open-addressing map uint64 -> uint32 (linear probing).  Key ~0 is empty. */
typedef struct {
    uint64_t *keys;
    uint32_t *vals;
    uint64_t mask;
} u64map;

static int u64map_init(u64map *m, uint64_t expected) {
    uint64_t cap = 64;
    while (cap < expected * 2) cap <<= 1;
    m->keys = (uint64_t *)malloc(cap * sizeof(uint64_t));
    m->vals = (uint32_t *)malloc(cap * sizeof(uint32_t));
    if (!m->keys || !m->vals) {
        free(m->keys);
        free(m->vals);
        return -1;
    }
    memset(m->keys, 0xff, cap * sizeof(uint64_t));
    m->mask = cap - 1;
    return 0;
}

static void u64map_free(u64map *m) {
    free(m->keys);
    free(m->vals);
}

static uint64_t mix64(uint64_t k) {
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdULL;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ULL;
    k ^= k >> 33;
    return k;
}

/* Returns a pointer to the value slot; *found tells whether it existed. */
static uint32_t *u64map_slot(u64map *m, uint64_t key, int *found) {
    uint64_t h = mix64(key) & m->mask;
    for (;;) {
        if (m->keys[h] == key) {
            *found = 1;
            return &m->vals[h];
        }
        if (m->keys[h] == ~0ULL) {
            m->keys[h] = key;
            *found = 0;
            return &m->vals[h];
        }
        h = (h + 1) & m->mask;
    }
}

/* ----------------------------------------------------------------- graph -- */

int64_t orc_ugraph_build(int64_t n_pairs, const uint32_t *src, const uint32_t *dst,
                         uint32_t *node_map_r, uint32_t *e_lo, uint32_t *e_hi,
                         int64_t *n_edges) {
    u64map nodes, edges;
    if (u64map_init(&nodes, (uint64_t)n_pairs * 2 + 1)) return -1;
    if (u64map_init(&edges, (uint64_t)n_pairs + 1)) {
        u64map_free(&nodes);
        return -1;
    }
    uint32_t node_count = 0;
    int64_t edge_count = 0;
    for (int64_t e = 0; e < n_pairs; ++e) {
        uint32_t s = src[e], t = dst[e];
        if (s == t) continue; /* RPGraph.cpp:52 */
        /* has_edge (:61-77) can only be true when both ends are known. */
        int fs, ft, fe;
        uint32_t *ps = u64map_slot(&nodes, s, &fs);
        uint32_t sm, tm;
        if (fs) {
            sm = *ps;
        } else {
            sm = node_count; /* add_node (:79-87): s first */
            *ps = sm;
            node_map_r[node_count++] = s;
        }
        uint32_t *pt = u64map_slot(&nodes, t, &ft);
        if (ft) {
            tm = *pt;
        } else {
            tm = node_count;
            *pt = tm;
            node_map_r[node_count++] = t;
        }
        uint32_t lo = sm < tm ? sm : tm, hi = sm < tm ? tm : sm;
        u64map_slot(&edges, ((uint64_t)lo << 32) | hi, &fe);
        if (fe) continue; /* duplicate undirected edge */
        e_lo[edge_count] = lo; /* adjacency_list[min].push_back(max) (:98) */
        e_hi[edge_count] = hi;
        edge_count++;
    }
    u64map_free(&nodes);
    u64map_free(&edges);
    *n_edges = edge_count;
    return node_count;
}

void orc_coo_order(int32_t n_nodes, int64_t n_edges, const uint32_t *e_lo,
                   const uint32_t *e_hi, int32_t *sources, int32_t *targets,
                   uint32_t *degree) {
    int64_t *start = (int64_t *)calloc((size_t)n_nodes + 1, sizeof(int64_t));
    memset(degree, 0, (size_t)n_nodes * sizeof(uint32_t));
    for (int64_t e = 0; e < n_edges; ++e) {
        start[e_lo[e] + 1]++;
        degree[e_lo[e]]++;
        degree[e_hi[e]]++;
    }
    for (int32_t i = 0; i < n_nodes; ++i) start[i + 1] += start[i];
    for (int64_t e = 0; e < n_edges; ++e) { /* stable by source */
        int64_t p = start[e_lo[e]]++;
        sources[p] = (int32_t)e_lo[e];
        targets[p] = (int32_t)e_hi[e];
    }
    free(start);
}

/* ---------------------------------------------------------------- layout -- */

static float get_random(float lowerbound, float upperbound) {
    /* RPCommon.cpp:50-53 */
    return lowerbound + (upperbound - lowerbound) * (float)random() / (float)RAND_MAX;
}

void orc_random_positions(int32_t n, float width, float height, uint32_t seed, float *xy) {
    srandom(seed);
    for (int32_t i = 0; i < n; ++i) {
        /* RPGraphLayout.cpp:49-50: the bounds are double expressions passed
         * to float parameters. */
        xy[2 * i] = get_random((float)(-width / 2.0), (float)(width / 2.0));
        xy[2 * i + 1] = get_random((float)(-height / 2.0), (float)(height / 2.0));
    }
}

/* ----------------------------------------------------------- FA2 kernels -- */

void orc_gravity(int32_t n, const float *xy, const float *mass, float k_g,
                 int32_t strong_gravity, float *fx, float *fy) {
    for (int32_t i = 0; i < n; ++i) {
        const float px = xy[2 * i], py = xy[2 * i + 1];
        float f_g;
        if (strong_gravity) {
            f_g = k_g * mass[i];
        } else if (px != 0.0 || py != 0.0) {
            /* rsqrtf of the kernel, written as 1/sqrtf. */
            f_g = k_g * mass[i] * (1.0f / sqrtf(px * px + py * py));
        } else {
            f_g = 0.0;
        }
        fx[i] += (-px * f_g);
        fy[i] += (-py * f_g);
    }
}

void orc_attraction(int64_t n_edges, const int32_t *sources, const int32_t *targets,
                    const float *xy, float *fx, float *fy) {
    for (int64_t e = 0; e < n_edges; ++e) {
        const int32_t s = sources[e], t = targets[e];
        const float dx = xy[2 * t] - xy[2 * s];
        const float dy = xy[2 * t + 1] - xy[2 * s + 1];
        fx[s] += dx;
        fy[s] += dy;
        fx[t] += -dx;
        fy[t] += -dy;
    }
}

/* Linear-log attraction, use_linlog in the reference's CPU path
 * (RPCPUForceAtlas2.cpp:55-78): per edge the distance vector p_t - p_s times
 * log(1 + d) / d, with d = 0 taken as FLT_MAX; added to s and subtracted
 * from t, in the edge order of the linear form above. */
void orc_attraction_linlog(int64_t n_edges, const int32_t *sources, const int32_t *targets,
                           const float *xy, float *fx, float *fy) {
    for (int64_t e = 0; e < n_edges; ++e) {
        const int32_t s = sources[e], t = targets[e];
        const float ex = xy[2 * s] - xy[2 * t];
        const float ey = xy[2 * s + 1] - xy[2 * t + 1];
        const float dist = sqrtf(ex * ex + ey * ey);
        const float w = dist == 0.0f ? FLT_MAX : logf(1 + dist) / dist;
        const float dx = xy[2 * t] - xy[2 * s];
        const float dy = xy[2 * t + 1] - xy[2 * s + 1];
        fx[s] += dx * w;
        fy[s] += dy * w;
        fx[t] += dx * -w;
        fy[t] += dy * -w;
    }
}

void orc_attraction_weighted(int64_t n_edges, const int32_t *sources, const int32_t *targets,
                             const float *wd, int32_t linlog, const float *xy, float *fx,
                             float *fy) {
    for (int64_t e = 0; e < n_edges; ++e) {
        const int32_t s = sources[e], t = targets[e];
        float w = 1.0f;
        if (linlog) {
            const float ex = xy[2 * s] - xy[2 * t];
            const float ey = xy[2 * s + 1] - xy[2 * t + 1];
            const float dist = sqrtf(ex * ex + ey * ey);
            w = dist == 0.0f ? FLT_MAX : logf(1 + dist) / dist;
        }
        float dx = xy[2 * t] - xy[2 * s];
        float dy = xy[2 * t + 1] - xy[2 * s + 1];
        if (linlog) {
            dx = dx * w;
            dy = dy * w;
        }
        dx = dx * wd[e];
        dy = dy * wd[e];
        fx[s] += dx;
        fy[s] += dy;
        fx[t] += -dx;
        fy[t] += -dy;
    }
}

void orc_speed_init(orc_speed_state *st) {
    st->global_speed = 1.0f;
    st->speed_efficiency = 1.0f;
    st->jitter_tolerance = 1.0f;
    st->k_s_max = 10.0f;
}

void orc_speed_update(int32_t n, float swg, float etra, orc_speed_state *st) {
    /* RPFA2Kernels.cu:177-219 */
    float estimated_optimal_jitter_tollerance = 0.05 * sqrtf((float)n);
    float minJT = sqrtf(estimated_optimal_jitter_tollerance);
    float jt = st->jitter_tolerance *
               fmaxf(minJT, fminf(st->k_s_max, estimated_optimal_jitter_tollerance * etra /
                                                   powf((float)n, 2.0f)));
    float min_speed_efficiency = 0.05;
    if (swg / etra > 2.0) {
        if (st->speed_efficiency > min_speed_efficiency) st->speed_efficiency *= 0.5;
        jt = fmaxf(jt, st->jitter_tolerance);
    }
    float targetSpeed = jt * st->speed_efficiency * etra / swg;
    if (swg > jt * etra) {
        if (st->speed_efficiency > min_speed_efficiency) st->speed_efficiency *= 0.7;
    } else if (st->global_speed < 1000) {
        st->speed_efficiency *= 1.3;
    }
    float max_rise = 0.5;
    st->global_speed += fminf(targetSpeed - st->global_speed, max_rise * st->global_speed);
}

void orc_speed(int32_t n, const float *fx, const float *fy, const float *fxp,
               const float *fyp, const float *mass, int32_t threads,
               orc_speed_state *st, float *swg_sum, float *etra_sum) {
    float *sswg = (float *)calloc((size_t)threads, sizeof(float));
    float *setra = (float *)calloc((size_t)threads, sizeof(float));
    for (int32_t t = 0; t < threads; ++t) { /* RPFA2Kernels.cu:131-148 */
        float swg_thread = 0, etra_thread = 0;
        for (int32_t j = t; j < n; j += threads) {
            float m = mass[j];
            float dx = fx[j] - fxp[j], dy = fy[j] - fyp[j];
            float swg_body = sqrtf(dx * dx + dy * dy);
            swg_thread += m * swg_body;
            dx = fx[j] + fxp[j];
            dy = fy[j] + fyp[j];
            float etra_body = sqrtf(dx * dx + dy * dy) / 2.0;
            etra_thread += m * etra_body;
        }
        sswg[t] = swg_thread;
        setra[t] = etra_thread;
    }
    for (int32_t j = threads / 2; j > 0; j /= 2) /* :151-160 */
        for (int32_t i = 0; i < j; ++i) {
            sswg[i] = sswg[i] + sswg[i + j];
            setra[i] = setra[i] + setra[i + j];
        }
    /* one block: the last-block sum (:175-182) is 0 + the block result */
    float swg = 0.0f + sswg[0], etra = 0.0f + setra[0];
    free(sswg);
    free(setra);
    orc_speed_update(n, swg, etra, st);
    if (swg_sum) *swg_sum = swg;
    if (etra_sum) *etra_sum = etra;
}

void orc_displacement(int32_t n, float *xy, float *fx, float *fy, float *fxp,
                      float *fyp, float global_speed) {
    for (int32_t i = 0; i < n; ++i) { /* RPFA2Kernels.cu:235-249 */
        float fxi = fx[i], fyi = fy[i];
        float dx = fxi - fxp[i], dy = fyi - fyp[i];
        float swg = sqrtf(dx * dx + dy * dy);
        float factor = global_speed / (1.0 + sqrtf(global_speed * swg));
        xy[2 * i] += fxi * factor;
        xy[2 * i + 1] += fyi * factor;
        fxp[i] = fxi;
        fyp[i] = fyi;
        fx[i] = 0.0;
        fy[i] = 0.0;
    }
}

/* ------------------------------------------------------------ Barnes-Hut -- */

struct orc_tree {
    int32_t n;            /* bodies */
    int32_t ncells, cap;  /* cell 0 is the root */
    int32_t *child;       /* 4 per cell: -1 empty, [0,n) body, n + c cell c */
    int32_t *depth;       /* tree depth of the cell: root 0, its children 1 */
    float *mass, *cx, *cy;
    int32_t *count;
    int32_t maxdepth;
    float radius, rootx, rooty;
};

static int32_t tree_new_cell(orc_tree *t, int32_t depth) {
    if (t->ncells == t->cap) {
        int32_t cap = t->cap * 2;
        int32_t *c = (int32_t *)realloc(t->child, (size_t)cap * 4 * sizeof(int32_t));
        int32_t *d = (int32_t *)realloc(t->depth, (size_t)cap * sizeof(int32_t));
        if (!c || !d) {
            if (c) t->child = c;
            if (d) t->depth = d;
            return -1;
        }
        t->child = c;
        t->depth = d;
        t->cap = cap;
    }
    int32_t k = t->ncells++;
    for (int i = 0; i < 4; ++i) t->child[4 * k + i] = -1;
    t->depth[k] = depth;
    return k;
}

orc_tree *orc_tree_build(int32_t n, float *xy, int32_t *n_perturbed) {
    orc_tree *t = (orc_tree *)calloc(1, sizeof(orc_tree));
    if (!t) return NULL;
    t->n = n;
    t->cap = n > 16 ? n : 16;
    t->child = (int32_t *)malloc((size_t)t->cap * 4 * sizeof(int32_t));
    t->depth = (int32_t *)malloc((size_t)t->cap * sizeof(int32_t));
    if (!t->child || !t->depth) {
        orc_tree_free(t);
        return NULL;
    }
    int32_t perturbed = 0;

    /* BoundingBoxKernel (RPBHKernels.cu:83-148) */
    float minx = xy[0], maxx = xy[0], miny = xy[1], maxy = xy[1];
    for (int32_t j = 0; j < n; ++j) {
        minx = fminf(minx, xy[2 * j]);
        maxx = fmaxf(maxx, xy[2 * j]);
        miny = fminf(miny, xy[2 * j + 1]);
        maxy = fmaxf(maxy, xy[2 * j + 1]);
    }
    t->radius = fmaxf(maxx - minx, maxy - miny) * 0.5f;
    t->rootx = (minx + maxx) * 0.5f;
    t->rooty = (miny + maxy) * 0.5f;
    tree_new_cell(t, 0);
    t->maxdepth = 1;

    const int32_t NB = n;
    for (int32_t i = 0; i < n; ++i) {
    restart:;
        /* TreeBuildingKernel (RPBHKernels.cu:209-243) */
        const float px = xy[2 * i], py = xy[2 * i + 1];
        int32_t node = 0, depth = 1, j = 0;
        float r = t->radius * 0.5f, dx = -r, dy = -r;
        if (t->rootx < px) { j = 1; dx = r; }
        if (t->rooty < py) { j |= 2; dy = r; }
        float x = t->rootx + dx, y = t->rooty + dy;
        int32_t ch = t->child[4 * node + j];
        while (ch >= NB) {
            node = ch - NB;
            depth++;
            r *= 0.5f;
            dx = dy = -r;
            j = 0;
            if (x < px) { j = 1; dx = r; }
            if (y < py) { j |= 2; dy = r; }
            x += dx;
            y += dy;
            ch = t->child[4 * node + j];
        }
        if (ch == -1) { /* :252-259 */
            t->child[4 * node + j] = i;
            if (depth > t->maxdepth) t->maxdepth = depth;
            continue;
        }
        /* a body is there (:262-319) */
        if (xy[2 * ch] == px && xy[2 * ch + 1] == py) {
            xy[2 * i] *= .99;
            xy[2 * i + 1] *= .99;
            perturbed++;
            goto restart;
        }
        int32_t slot = 4 * node + j;
        do {
            int32_t cell = tree_new_cell(t, depth);
            if (cell < 0) {
                orc_tree_free(t);
                return NULL;
            }
            t->child[slot] = NB + cell;
            depth++;
            node = cell;
            r *= 0.5f;
            j = 0;
            if (x < xy[2 * ch]) j = 1;
            if (y < xy[2 * ch + 1]) j |= 2;
            t->child[4 * cell + j] = ch;
            j = 0;
            dx = dy = -r;
            if (x < px) { j = 1; dx = r; }
            if (y < py) { j |= 2; dy = r; }
            x += dx;
            y += dy;
            slot = 4 * node + j;
        } while (t->child[slot] >= 0);
        t->child[slot] = i;
        if (depth > t->maxdepth) t->maxdepth = depth;
    }
    if (n_perturbed) *n_perturbed = perturbed;
    t->mass = (float *)calloc((size_t)t->ncells, sizeof(float));
    t->cx = (float *)calloc((size_t)t->ncells, sizeof(float));
    t->cy = (float *)calloc((size_t)t->ncells, sizeof(float));
    t->count = (int32_t *)calloc((size_t)t->ncells, sizeof(int32_t));
    if (!t->mass || !t->cx || !t->cy || !t->count) {
        orc_tree_free(t);
        return NULL;
    }
    return t;
}

void orc_tree_free(orc_tree *t) {
    if (!t) return;
    free(t->child);
    free(t->depth);
    free(t->mass);
    free(t->cx);
    free(t->cy);
    free(t->count);
    free(t);
}

int32_t orc_tree_maxdepth(const orc_tree *t) { return t->maxdepth; }
float orc_tree_radius(const orc_tree *t) { return t->radius; }
int32_t orc_tree_num_cells(const orc_tree *t) { return t->ncells; }
void orc_tree_root(const orc_tree *t, float *cx, float *cy) {
    *cx = t->rootx;
    *cy = t->rooty;
}

void orc_tree_summarize(orc_tree *t, const float *xy, const float *mass) {
    /* A cell is always created before its sub-cells, so a reverse sweep over
     * cell ids visits children first (the order the kernel's waits enforce). */
    const int32_t NB = t->n;
    for (int32_t k = t->ncells - 1; k >= 0; --k) { /* RPBHKernels.cu:461-494 */
        float cm = 0.0f, px = 0.0f, py = 0.0f, m;
        int32_t cnt = 0;
        for (int i = 0; i < 4; ++i) {
            int32_t ch = t->child[4 * k + i];
            if (ch < 0) continue;
            if (ch >= NB) {
                int32_t c = ch - NB;
                m = t->mass[c];
                cnt += t->count[c];
                px += t->cx[c] * m;
                py += t->cy[c] * m;
            } else {
                m = mass[ch];
                cnt++;
                px += xy[2 * ch] * m;
                py += xy[2 * ch + 1] * m;
            }
            cm += m;
        }
        t->count[k] = cnt;
        m = 1.0f / cm;
        t->cx[k] = px * m;
        t->cy[k] = py * m;
        t->mass[k] = cm;
    }
}

/* Depth-first walk, children in quadrant order; calls back on cells and bodies. */
typedef struct {
    int32_t node;
    int32_t pd;
} walk_frame;

void orc_tree_sort(const orc_tree *t, int32_t *sortd) {
    const int32_t NB = t->n;
    walk_frame *st = (walk_frame *)malloc((size_t)(t->ncells + 1) * sizeof(walk_frame));
    int32_t sp = 0, out = 0;
    st[sp++] = (walk_frame){0, 0};
    while (sp > 0) {
        walk_frame *f = &st[sp - 1];
        if (f->pd == 4) {
            sp--;
            continue;
        }
        int32_t ch = t->child[4 * f->node + f->pd++];
        if (ch < 0) continue;
        if (ch >= NB)
            st[sp++] = (walk_frame){ch - NB, 0};
        else
            sortd[out++] = ch; /* SortKernel :548-553 */
    }
    free(st);
}

void orc_tree_cells(const orc_tree *t, int32_t *level, float *mass, float *cx,
                    float *cy, int32_t *count) {
    const int32_t NB = t->n;
    walk_frame *st = (walk_frame *)malloc((size_t)(t->ncells + 1) * sizeof(walk_frame));
    int32_t sp = 0, out = 0;
    st[sp++] = (walk_frame){0, 0};
    level[out] = 0;
    mass[out] = t->mass[0];
    cx[out] = t->cx[0];
    cy[out] = t->cy[0];
    count[out] = t->count[0];
    out++;
    while (sp > 0) {
        walk_frame *f = &st[sp - 1];
        if (f->pd == 4) {
            sp--;
            continue;
        }
        int32_t ch = t->child[4 * f->node + f->pd++];
        if (ch < NB) continue;
        int32_t c = ch - NB;
        level[out] = t->depth[c];
        mass[out] = t->mass[c];
        cx[out] = t->cx[c];
        cy[out] = t->cy[c];
        count[out] = t->count[c];
        out++;
        st[sp++] = (walk_frame){c, 0};
    }
    free(st);
}

#define ORC_MAXDEPTH 32 /* RPBHFA2LaunchParameters.cuh:62 */

/* prevent_overlap (RPForceAtlas2.hpp:44; the reference declares it and its
 * CPU displacement exits with "Not yet implemented", RPCPUForceAtlas2.cpp:
 * 201-205).  The rule of the ForceAtlas2 paper (Jacomy et al., PLoS ONE
 * 2014), with d' = d - s_i - s_j the border-to-border distance: repulsion
 * k_r m_i m_j / d' while the nodes are apart, k_r' m_i m_j with k_r' = 100 k_r
 * while they overlap, nothing at d' = 0; attraction d' while apart, nothing
 * while they overlap.  Applied between bodies; a Barnes-Hut cell, which has
 * no size, repels as a point mass.  d is the walk's softened distance
 * sqrt(d^2 + eps).  Returns the factor c with force = k_r m_i c (p_i - p_j). */
static float overlap_factor(float d2, float si, float sj, float mj) {
    const float ds = sqrtf(d2);
    const float dp = ds - si - sj;
    if (dp > 0.0f) return mj / (ds * dp);
    if (dp < 0.0f) return 100.0f * mj / ds;
    return 0.0f;
}

void orc_attraction_overlap(int64_t n_edges, const int32_t *sources, const int32_t *targets,
                            const float *sizes, const float *xy, float *fx, float *fy) {
    for (int64_t e = 0; e < n_edges; ++e) {
        const int32_t s = sources[e], t = targets[e];
        const float dx = xy[2 * t] - xy[2 * s];
        const float dy = xy[2 * t + 1] - xy[2 * s + 1];
        const float d = sqrtf(dx * dx + dy * dy);
        const float dp = d - sizes[s] - sizes[t];
        const float w = dp > 0.0f ? dp / d : 0.0f;
        const float qx = dx * w, qy = dy * w;
        fx[s] += qx;
        fy[s] += qy;
        fx[t] += -qx;
        fy[t] += -qy;
    }
}

/* The walk of ForceCalculationKernel (restated below); with a2r/a2i set, each
 * accepted cell also adds its quadrupole term (orc_tree_repulsion_quad). */
static int32_t tree_walk(const orc_tree *t, const float *xy, const float *mass, float k_r,
                         float itolsq, float epssq, int32_t group, const int32_t *sortd,
                         const double *a2r, const double *a2i, const float *sizes, float *fx,
                         float *fy, int64_t *n_visits) {
    const int32_t NB = t->n;
    if (n_visits) *n_visits = 0;
    if (t->maxdepth > ORC_MAXDEPTH) return 1; /* RPBHKernels.cu:595 */

    /* dq table, RPBHKernels.cu:579-592 */
    float dq[ORC_MAXDEPTH];
    float tmp = t->radius * 2;
    dq[0] = tmp * tmp * itolsq;
    int32_t i;
    for (i = 1; i < t->maxdepth; i++) {
        dq[i] = dq[i - 1] * 0.25f;
        dq[i - 1] += epssq;
    }
    dq[i - 1] += epssq;

    int32_t *lane_body = (int32_t *)malloc((size_t)group * sizeof(int32_t));
    float *ax = (float *)malloc((size_t)group * sizeof(float));
    float *ay = (float *)malloc((size_t)group * sizeof(float));
    int32_t stack_node[ORC_MAXDEPTH + 1], stack_pd[ORC_MAXDEPTH + 1];
    int64_t visits = 0;

    for (int32_t base = 0; base < NB; base += group) {
        int32_t lanes = NB - base < group ? NB - base : group;
        for (int32_t l = 0; l < lanes; ++l) {
            lane_body[l] = sortd[base + l];
            ax[l] = 0.0f;
            ay[l] = 0.0f;
        }
        /* :621-685 */
        int32_t depth = 0;
        stack_node[0] = 0;
        stack_pd[0] = 0;
        do {
            int32_t pd = stack_pd[depth], nd = stack_node[depth];
            while (pd < 4) {
                int32_t n = t->child[4 * nd + pd];
                pd++;
                if (n < 0) continue; /* compacted children end early; same set */
                float nx, ny, nm;
                if (n < NB) {
                    nx = xy[2 * n];
                    ny = xy[2 * n + 1];
                    nm = mass[n];
                } else {
                    nx = t->cx[n - NB];
                    ny = t->cy[n - NB];
                    nm = t->mass[n - NB];
                }
                int all = 1;
                if (n >= NB) {
                    for (int32_t l = 0; l < lanes; ++l) {
                        const int32_t b = lane_body[l];
                        const float dx = xy[2 * b] - nx, dy = xy[2 * b + 1] - ny;
                        const float d2 = dx * dx + dy * dy + epssq;
                        if (!(d2 >= dq[depth])) {
                            all = 0;
                            break;
                        }
                    }
                }
                visits += lanes;
                if (all) {
                    for (int32_t l = 0; l < lanes; ++l) {
                        const int32_t b = lane_body[l];
                        const float dx = xy[2 * b] - nx, dy = xy[2 * b + 1] - ny;
                        const float d2 = dx * dx + dy * dy + epssq;
                        if (sizes && n < NB) {
                            /* prevent_overlap: border-to-border distance */
                            const float c = overlap_factor(d2, sizes[b], sizes[n], nm);
                            ax[l] += k_r * dx * mass[b] * c;
                            ay[l] += k_r * dy * mass[b] * c;
                            continue;
                        }
                        ax[l] += k_r * dx * mass[b] * nm / d2;
                        ay[l] += k_r * dy * mass[b] * nm / d2;
                        if (a2r && n >= NB) {
                            /* conj(a2 / w^3) = conj(a2 conj(w)^3) / |w|^6, |w|^2 = d2 */
                            const double qr = a2r[n - NB], qi = a2i[n - NB];
                            const double ur = (double)dx * ((double)dx * dx - 3.0 * dy * dy);
                            const double ui = (double)dy * ((double)dy * dy - 3.0 * dx * dx);
                            const double inv = 1.0 / ((double)d2 * d2 * d2);
                            ax[l] += (float)(k_r * mass[b] * (qr * ur - qi * ui) * inv);
                            ay[l] += (float)(-k_r * mass[b] * (qr * ui + qi * ur) * inv);
                        }
                    }
                } else {
                    stack_pd[depth] = pd;
                    stack_node[depth] = nd;
                    depth++;
                    pd = 0;
                    nd = n - NB;
                }
            }
            depth--;
        } while (depth >= 0);
        for (int32_t l = 0; l < lanes; ++l) { /* :689-690 */
            fx[lane_body[l]] += ax[l];
            fy[lane_body[l]] += ay[l];
        }
    }
    free(lane_body);
    free(ax);
    free(ay);
    if (n_visits) *n_visits = visits;
    return 0;
}

int32_t orc_tree_repulsion(const orc_tree *t, const float *xy, const float *mass,
                           float k_r, float itolsq, float epssq, int32_t group,
                           const int32_t *sortd, float *fx, float *fy,
                           int64_t *n_visits) {
    return tree_walk(t, xy, mass, k_r, itolsq, epssq, group, sortd, NULL, NULL, NULL, fx, fy,
                     n_visits);
}

int32_t orc_tree_repulsion_overlap(const orc_tree *t, const float *xy, const float *mass,
                                   const float *sizes, float k_r, float itolsq, float epssq,
                                   int32_t group, const int32_t *sortd, float *fx, float *fy,
                                   int64_t *n_visits) {
    return tree_walk(t, xy, mass, k_r, itolsq, epssq, group, sortd, NULL, NULL, sizes, fx, fy,
                     n_visits);
}

/* Quadrupole extension, no reference counterpart: the complex second moment
 * a2 = sum m (z - Z)^2 of every cell about its centre of mass, bottom-up over
 * the children with the parallel-axis rule. */
static void cell_quadrupoles(const orc_tree *t, const float *xy, const float *mass, int32_t c,
                             double *a2r, double *a2i) {
    const int32_t NB = t->n;
    double sr = 0.0, si = 0.0;
    for (int q = 0; q < 4; ++q) {
        const int32_t ch = t->child[4 * c + q];
        if (ch < 0) continue;
        double mx, my, m, cr = 0.0, ci = 0.0;
        if (ch < NB) {
            mx = xy[2 * ch];
            my = xy[2 * ch + 1];
            m = mass[ch];
        } else {
            cell_quadrupoles(t, xy, mass, ch - NB, a2r, a2i);
            mx = t->cx[ch - NB];
            my = t->cy[ch - NB];
            m = t->mass[ch - NB];
            cr = a2r[ch - NB];
            ci = a2i[ch - NB];
        }
        const double dx = mx - t->cx[c], dy = my - t->cy[c];
        sr += cr + m * (dx * dx - dy * dy);
        si += ci + m * (2.0 * dx * dy);
    }
    a2r[c] = sr;
    a2i[c] = si;
}

int32_t orc_tree_repulsion_quad(const orc_tree *t, const float *xy, const float *mass,
                                float k_r, float itolsq, float epssq, int32_t group,
                                const int32_t *sortd, float *fx, float *fy, int64_t *n_visits) {
    if (t->maxdepth > ORC_MAXDEPTH) return 1;
    double *a2r = (double *)calloc((size_t)t->ncells + 1, sizeof(double));
    double *a2i = (double *)calloc((size_t)t->ncells + 1, sizeof(double));
    if (!a2r || !a2i) {
        free(a2r);
        free(a2i);
        return -1;
    }
    cell_quadrupoles(t, xy, mass, 0, a2r, a2i);
    int32_t r = tree_walk(t, xy, mass, k_r, itolsq, epssq, group, sortd, a2r, a2i, NULL, fx, fy,
                          n_visits);
    free(a2r);
    free(a2i);
    return r;
}

typedef struct {
    int32_t n;
    const float *xy, *mass;
    double k_r, eps;
    int32_t n_samples;
    const int32_t *samples;
    double *fx, *fy;
    int32_t *next; /* shared work counter */
    pthread_mutex_t *lock;
} exact_job;

static void *exact_worker(void *arg) {
    exact_job *jb = (exact_job *)arg;
    for (;;) {
        pthread_mutex_lock(jb->lock);
        int32_t s0 = *jb->next;
        *jb->next += 8;
        pthread_mutex_unlock(jb->lock);
        if (s0 >= jb->n_samples) break;
        int32_t s1 = s0 + 8 < jb->n_samples ? s0 + 8 : jb->n_samples;
        for (int32_t s = s0; s < s1; ++s) {
            const int32_t i = jb->samples[s];
            const double px = jb->xy[2 * i], py = jb->xy[2 * i + 1], mi = jb->mass[i];
            double ax = 0.0, ay = 0.0;
            for (int32_t j = 0; j < jb->n; ++j) {
                if (j == i) continue;
                const double dx = px - (double)jb->xy[2 * j], dy = py - (double)jb->xy[2 * j + 1];
                const double d2 = dx * dx + dy * dy + jb->eps;
                if (d2 == 0.0) continue;
                const double f = jb->k_r * mi * (double)jb->mass[j] / d2;
                ax += dx * f;
                ay += dy * f;
            }
            jb->fx[s] = ax;
            jb->fy[s] = ay;
        }
    }
    return NULL;
}

void orc_exact_repulsion_f64(int32_t n, const float *xy, const float *mass, double k_r,
                             double eps, int32_t n_samples, const int32_t *samples,
                             double *fx, double *fy) {
    long ncpu = sysconf(_SC_NPROCESSORS_ONLN);
    int32_t nthreads = ncpu < 1 ? 1 : (ncpu > 64 ? 64 : (int32_t)ncpu);
    int32_t next = 0;
    pthread_mutex_t lock = PTHREAD_MUTEX_INITIALIZER;
    exact_job jb = {n, xy, mass, k_r, eps, n_samples, samples, fx, fy, &next, &lock};
    pthread_t th[64];
    for (int32_t t = 1; t < nthreads; ++t) pthread_create(&th[t], NULL, exact_worker, &jb);
    exact_worker(&jb);
    for (int32_t t = 1; t < nthreads; ++t) pthread_join(th[t], NULL);
}

/* ------------------------------------------------------------- full step -- */

int32_t orc_fa2_step(orc_fa2 *s) {
    const int32_t n = s->n;
    /* fx, fy are zero here: the previous displacement cleared them. */
    orc_gravity(n, s->xy, s->mass, s->k_g, s->strong_gravity, s->fx, s->fy);
    if (s->sizes)
        orc_attraction_overlap(s->m, s->sources, s->targets, s->sizes, s->xy, s->fx, s->fy);
    else if (s->linlog)
        orc_attraction_linlog(s->m, s->sources, s->targets, s->xy, s->fx, s->fy);
    else
        orc_attraction(s->m, s->sources, s->targets, s->xy, s->fx, s->fy);
    if (s->f_ga_out)
        for (int32_t i = 0; i < n; ++i) {
            s->f_ga_out[2 * i] = s->fx[i];
            s->f_ga_out[2 * i + 1] = s->fy[i];
        }
    orc_tree *t = orc_tree_build(n, s->xy, &s->n_perturbed);
    if (!t) return -1;
    orc_tree_summarize(t, s->xy, s->mass);
    int32_t *sortd = s->sortd_out ? s->sortd_out : (int32_t *)malloc((size_t)n * sizeof(int32_t));
    orc_tree_sort(t, sortd);
    /* maxdepthd is never reset between steps (RPBHKernels.cu:59, :328), so
     * once a tree is deeper than 32 levels the force kernel stays off. */
    if (t->maxdepth > s->maxdepth) s->maxdepth = t->maxdepth;
    s->depth_overflow = s->maxdepth > ORC_MAXDEPTH;
    if (!s->depth_overflow)
        tree_walk(t, s->xy, s->mass, s->k_r, s->itolsq, s->epssq, s->group, sortd, NULL, NULL,
                  s->sizes, s->fx, s->fy, NULL);
    if (!s->sortd_out) free(sortd);
    orc_tree_free(t);
    if (s->f_tot_out)
        for (int32_t i = 0; i < n; ++i) {
            s->f_tot_out[2 * i] = s->fx[i];
            s->f_tot_out[2 * i + 1] = s->fy[i];
        }
    orc_speed(n, s->fx, s->fy, s->fxp, s->fyp, s->mass, s->speed_threads, &s->speed,
              &s->swg_sum, &s->etra_sum);
    orc_displacement(n, s->xy, s->fx, s->fy, s->fxp, s->fyp, s->speed.global_speed);
    return 0;
}
