/*
 * ref_cpu_harness.cpp -- a C interface over the reference's own host classes
 * (RPGraph::UGraph, GraphLayout, CPUForceAtlas2), linked from the reference
 * sources at build time.  TEST INFRASTRUCTURE ONLY: it pins the oracle's graph
 * build and FA2 update rules, and it is the timed CPU baseline of bench.py.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <string>
#include <unordered_map>
#include <vector>

// The harness reads the classes' private state (forces, speed) directly.
#define private public
#define protected public
#include "RPCPUForceAtlas2.hpp"
#include "RPGraph.hpp"
#include "RPGraphLayout.hpp"
#undef private
#undef protected

using namespace RPGraph;

namespace {
struct RefFa2 {
    GraphLayout *layout;
    CPUForceAtlas2 *fa2;
};
}  // namespace

extern "C" {

void *refcpu_load(const char *path) { return new UGraph(std::string(path)); }

/* A UGraph holding the given nodes and edges, filled into the reference's own
 * members the way add_node/add_edge (RPGraph.cpp:79-102) would fill them from
 * an edge list, without re-reading a file (the reference's loader copies a
 * neighbour list per line and takes minutes on large graphs).  e_lo/e_hi are
 * the mapped (min, max) edge ends in file order. */
void *refcpu_graph_from_arrays(uint32_t n_nodes, const uint32_t *node_map_r, uint64_t n_edges,
                               const uint32_t *e_lo, const uint32_t *e_hi) {
    UGraph *g = new UGraph(std::string("/nonexistent/fa2-empty-edgelist"));
    g->node_count = n_nodes;
    g->edge_count = (nid_t)n_edges;
    g->node_map.reserve(n_nodes);
    g->node_map_r.reserve(n_nodes);
    for (nid_t n = 0; n < n_nodes; ++n) {
        g->node_map[node_map_r[n]] = n;
        g->node_map_r[n] = node_map_r[n];
    }
    for (uint64_t e = 0; e < n_edges; ++e) {
        g->adjacency_list[e_lo[e]].push_back(e_hi[e]);
        g->degrees[e_lo[e]] += 1;
        g->degrees[e_hi[e]] += 1;
    }
    return g;
}
void refcpu_free_graph(void *g) { delete (UGraph *)g; }
uint32_t refcpu_num_nodes(void *g) { return ((UGraph *)g)->num_nodes(); }
uint32_t refcpu_num_edges(void *g) { return ((UGraph *)g)->num_edges(); }

void refcpu_node_map_r(void *gp, uint32_t *out) {
    UGraph *g = (UGraph *)gp;
    for (nid_t n = 0; n < g->num_nodes(); ++n) out[n] = g->node_map_r[n];
}

void refcpu_degrees(void *gp, uint32_t *out) {
    UGraph *g = (UGraph *)gp;
    for (nid_t n = 0; n < g->num_nodes(); ++n) out[n] = g->degree(n);
}

/* neighbors_with_geq_id of every node, concatenated; offsets has N+1 entries. */
void refcpu_adjacency(void *gp, uint32_t *offsets, uint32_t *adj) {
    UGraph *g = (UGraph *)gp;
    uint32_t k = 0;
    for (nid_t n = 0; n < g->num_nodes(); ++n) {
        offsets[n] = k;
        for (nid_t t : g->neighbors_with_geq_id(n)) adj[k++] = t;
    }
    offsets[g->num_nodes()] = k;
}

/* srandom(seed) as graph_viewer.cpp:49 does, then GraphLayout(graph, w, h) and
 * a CPUForceAtlas2, whose constructor randomizes the positions. */
void *refcpu_fa2_create(void *gp, float w, float h, uint32_t seed, int use_bh, int strong_gravity,
                        float gravity, float scale) {
    srandom(seed);
    RefFa2 *r = new RefFa2();
    r->layout = new GraphLayout(*(UGraph *)gp, w, h);
    r->fa2 = new CPUForceAtlas2(*r->layout, use_bh != 0, strong_gravity != 0, gravity, scale);
    return r;
}

void refcpu_fa2_destroy(void *p) {
    RefFa2 *r = (RefFa2 *)p;
    delete r->fa2;
    delete r->layout;
    delete r;
}

void refcpu_fa2_positions(void *p, float *xy) {
    RefFa2 *r = (RefFa2 *)p;
    for (nid_t n = 0; n < r->layout->graph.num_nodes(); ++n) {
        xy[2 * n] = r->layout->getX(n);
        xy[2 * n + 1] = r->layout->getY(n);
    }
}

void refcpu_fa2_set_positions(void *p, const float *xy) {
    RefFa2 *r = (RefFa2 *)p;
    for (nid_t n = 0; n < r->layout->graph.num_nodes(); ++n) {
        r->layout->setX(n, xy[2 * n]);
        r->layout->setY(n, xy[2 * n + 1]);
    }
}

void refcpu_fa2_step(void *p, int iters) {
    RefFa2 *r = (RefFa2 *)p;
    for (int i = 0; i < iters; ++i) r->fa2->doStep();
}

float refcpu_fa2_global_speed(void *p) { return ((RefFa2 *)p)->fa2->global_speed; }
float refcpu_fa2_speed_efficiency(void *p) { return ((RefFa2 *)p)->fa2->speed_efficiency; }

/* The force terms of CPUForceAtlas2::doStep (RPCPUForceAtlas2.cpp:226-237)
 * on the current positions, without moving anything: gravity + attraction,
 * and repulsion, each summed into a cleared force array. */
void refcpu_fa2_forces(void *p, float *f_ga, float *f_rep) {
    RefFa2 *r = (RefFa2 *)p;
    CPUForceAtlas2 *f = r->fa2;
    nid_t n_nodes = r->layout->graph.num_nodes();
    for (nid_t n = 0; n < n_nodes; ++n) f->forces[n] = Real2DVector(0.0f, 0.0f);
    for (nid_t n = 0; n < n_nodes; ++n) {
        f->apply_gravity(n);
        f->apply_attract(n);
    }
    for (nid_t n = 0; n < n_nodes; ++n) {
        f_ga[2 * n] = f->forces[n].x;
        f_ga[2 * n + 1] = f->forces[n].y;
        f->forces[n] = Real2DVector(0.0f, 0.0f);
    }
    if (f->use_barneshut) f->rebuild_bh();
    for (nid_t n = 0; n < n_nodes; ++n) f->apply_repulsion(n);
    for (nid_t n = 0; n < n_nodes; ++n) {
        f_rep[2 * n] = f->forces[n].x;
        f_rep[2 * n + 1] = f->forces[n].y;
        f->forces[n] = Real2DVector(0.0f, 0.0f);
    }
}

/* Stores forces and previous forces, so that refcpu_fa2_update_speeds runs
 * the reference's speed rule (CPUForceAtlas2::updateSpeeds,
 * RPCPUForceAtlas2.cpp:144-197) on them. */
void refcpu_fa2_set_forces(void *p, const float *f, const float *f_prev) {
    RefFa2 *r = (RefFa2 *)p;
    nid_t n_nodes = r->layout->graph.num_nodes();
    for (nid_t n = 0; n < n_nodes; ++n) {
        r->fa2->forces[n] = Real2DVector(f[2 * n], f[2 * n + 1]);
        r->fa2->prev_forces[n] = Real2DVector(f_prev[2 * n], f_prev[2 * n + 1]);
    }
}

void refcpu_fa2_update_speeds(void *p) { ((RefFa2 *)p)->fa2->updateSpeeds(); }

/* ForceAtlas2::use_linlog, public in the reference (RPForceAtlas2.hpp:44). */
void refcpu_fa2_set_linlog(void *p, int on) { ((RefFa2 *)p)->fa2->use_linlog = on != 0; }

/* GraphLayout::writeToCSV / writeToBin (RPGraphLayout.cpp:209-250). */
void refcpu_fa2_write(void *p, const char *path, int binary) {
    RefFa2 *r = (RefFa2 *)p;
    if (binary)
        r->layout->writeToBin(std::string(path));
    else
        r->layout->writeToCSV(std::string(path));
}

}  // extern "C"
