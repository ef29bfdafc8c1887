// fa2_capi.cu -- the C ABI of include/fa2b200.h: context set-up, the CUDA
// graph of one iteration, and the host side of the rare replay path.
//
// One iteration is captured once into a CUDA graph on two streams (attraction
// overlaps the tree build) and replayed per step.  When the tree build finds
// bodies at exactly the same position it flags the iteration ("poison") and
// every later kernel of the launch skips its work; the host then applies the
// reference's .99 scaling (src/RPBHKernels.cu:271-278) and re-runs that
// iteration from the key stage, before continuing with the rest.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <numeric>
#include <random>
#include <vector>

#include "../../include/fa2b200.h"
#include "fa2_internal.cuh"
#include "fa2_learn.cuh"

using namespace fa2;

namespace {

constexpr int kNumSlots = 10;
const char *const kSlotNames[kNumSlots] = {"attract",  "keys",     "sort",    "tree_count",
                                           "emit",     "traverse", "displace", "moments",
                                           "quadrupole", "learn"};
enum Slot { S_ATTRACT, S_KEYS, S_SORT, S_COUNT, S_EMIT, S_TRAV, S_DISP, S_MOM, S_QUAD, S_LEARN };

// The last CUDA error a call of this thread met, with the source line that saw
// it (fa2_last_cuda_error).
thread_local char g_last_cuda_error[192] = "";

constexpr int kMaxReplayRounds = 64;

}  // namespace

struct fa2_ctx {
    int device = 0;
    int nsm = 148;
    uint32_t n = 0;
    uint64_t m = 0;
    fa2_params prm{};
    Params kp{};
    std::vector<uint32_t> ref_of;  // internal -> reference id
    uint64_t nnz_pad = 0;
    AttractPlan plan{};
    Buffers b{};
    // allocations
    std::vector<void *> allocs;
    void *scratch = nullptr;
    size_t scratch_bytes = 0;
    float2 *stage_xy = nullptr;    // n, reference order
    DevState *h_state = nullptr;   // pinned: the state after fa2_step_host's iterations
    int *h_iters = nullptr;        // pinned: iterations done before them
    uint32_t *stage_ids = nullptr; // n
    int bbox_blocks = 0, trav_blocks = 0;
    cudaStream_t sA = nullptr, sB = nullptr;
    cudaEvent_t evFork = nullptr, evJoin = nullptr, evCounted = nullptr;
    cudaEvent_t evEmitted = nullptr, evA2 = nullptr;  // the learned cells' a2 pass on stream B
    // graphs
    cudaGraphExec_t exec = nullptr;
    cudaGraphExec_t exec_timed = nullptr;
    cudaGraph_t graph_timed = nullptr;         // kept: its nodes address exec_timed
    std::vector<cudaGraphNode_t> timed_nodes;  // event-record nodes, [slot*2 + start/end]
    std::vector<cudaEvent_t> slot_events;      // events captured into the timed graph
    std::vector<cudaEvent_t> event_pool;       // per (iteration, slot, start/end)
    int last_perturb_rounds = 0;
    bool overlap = true;  // attraction on stream B beside the tree build
    // accuracy guard (fa2_set_accuracy_guard)
    int guard_every = 0, guard_samples = 0, guard_cap = 0, guard_left = 0;
    int guard_checks = 0, guard_fallbacks = 0;
    double guard_err_cur = 0.0, guard_err_plain = 0.0;
    double2 *guard_exact = nullptr, *guard_part = nullptr;
    float2 *guard_plain = nullptr, *guard_cur = nullptr;
    // learned correction (fa2_set_learned_correction)
    bool learn_on = false;
    LearnBuffers lb{};
    MlpDevice *d_mlp = nullptr;
};

namespace {

// Drops the captured iteration graphs; the next step captures them again.
void drop_graphs(fa2_ctx *c) {
    if (c->exec) cudaGraphExecDestroy(c->exec);
    if (c->exec_timed) cudaGraphExecDestroy(c->exec_timed);
    if (c->graph_timed) cudaGraphDestroy(c->graph_timed);
    c->exec = c->exec_timed = nullptr;
    c->graph_timed = nullptr;
}

int cuda_status_at(cudaError_t e, int line) {
    if (e == cudaSuccess) return FA2_OK;
    snprintf(g_last_cuda_error, sizeof(g_last_cuda_error), "%s (%s) at fa2_capi.cu:%d",
             cudaGetErrorName(e), cudaGetErrorString(e), line);
    if (e == cudaErrorMemoryAllocation) return FA2_ERR_OUT_OF_MEMORY;
    return FA2_ERR_CUDA;
}
#define cuda_status(e) cuda_status_at((e), __LINE__)

#define CK(call)                                   \
    do {                                           \
        cudaError_t e_ = (call);                   \
        if (e_ != cudaSuccess) return cuda_status(e_); \
    } while (0)

template <typename T>
int dalloc(fa2_ctx *c, T **p, size_t count) {
    void *q = nullptr;
    size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
    CK(cudaMalloc(&q, bytes));
    c->allocs.push_back(q);
    *p = (T *)q;
    return FA2_OK;
}

// Buffers of the quadrupole option, allocated when it is first selected.
int ensure_quad_buffers(fa2_ctx *c) {
    Buffers &b = c->b;
    int s = FA2_OK;
    if ((!b.quad && (s = dalloc(c, &b.quad, b.capacity))) ||
        (!b.pmom && (s = dalloc(c, &b.pmom, (size_t)b.n + 1))) ||
        (!b.mom_lb && (s = dalloc(c, &b.mom_lb, (size_t)mom_tiles(b.n)))) ||
        (!b.mom_m && (s = dalloc(c, &b.mom_m, (size_t)b.n))) ||
        (!b.mom_q && (s = dalloc(c, &b.mom_q, (size_t)b.n))))
        return s;
    return FA2_OK;
}

// Buffers of the learned correction, allocated when it is first used: the
// pair list (up to 32 pairs per body), the groups' geometry and corrections,
// the sorted bodies' repulsion, the cells' second moments and the MLP's
// weights.
int ensure_learn_buffers(fa2_ctx *c) {
    LearnBuffers &lb = c->lb;
    const size_t groups = ((size_t)c->n + 31) / 32;
    // 32 pairs per body on average (a group accepts a few hundred cells at
    // theta >= 1), in kPairSegments segments with room for imbalance
    const uint64_t seg = std::min<uint64_t>((32ull * c->n) / kPairSegments + 4096, 0x7FFFFFFFull);
    const uint64_t cap = seg * kPairSegments;
    int s = FA2_OK;
    if ((!lb.pairs && (s = dalloc(c, &lb.pairs, (size_t)cap))) ||
        (!lb.ggeo && (s = dalloc(c, &lb.ggeo, 2 * groups))) ||
        (!lb.rep && (s = dalloc(c, &lb.rep, (size_t)c->n))) ||
        (!lb.corr && (s = dalloc(c, &lb.corr, groups))) ||
        (!lb.a2 && (s = dalloc(c, &lb.a2, c->b.capacity))) ||
        (!c->d_mlp && (s = dalloc(c, &c->d_mlp, 1))))
        return s;
    lb.seg_cap = (uint32_t)seg;
    lb.mlp = c->d_mlp;
    return FA2_OK;
}

void free_all(fa2_ctx *c) {
    if (c->exec) cudaGraphExecDestroy(c->exec);
    if (c->exec_timed) cudaGraphExecDestroy(c->exec_timed);
    if (c->graph_timed) cudaGraphDestroy(c->graph_timed);
    for (cudaEvent_t e : c->slot_events) cudaEventDestroy(e);
    for (cudaEvent_t e : c->event_pool) cudaEventDestroy(e);
    for (void *p : c->allocs) cudaFree(p);
    c->allocs.clear();
    if (c->evFork) cudaEventDestroy(c->evFork);
    if (c->evJoin) cudaEventDestroy(c->evJoin);
    if (c->evCounted) cudaEventDestroy(c->evCounted);
    if (c->evEmitted) cudaEventDestroy(c->evEmitted);
    if (c->evA2) cudaEventDestroy(c->evA2);
    if (c->sA) cudaStreamDestroy(c->sA);
    if (c->sB) cudaStreamDestroy(c->sB);
    if (c->h_state) cudaFreeHost(c->h_state);
    if (c->h_iters) cudaFreeHost(c->h_iters);
}

// Nodes in degree-descending order (ties by reference id), a symmetric CSR
// over that order with each row sorted and padded with its own id to a
// multiple of four, and the attraction buckets over it.
// The symmetric CSR in internal ids (degree order), rows sorted by
// neighbour id and padded with the row's own id to a multiple of four.  With
// `delta` != 0 and edge weights, wcol holds w^delta beside each entry
// (rounded once from double; 1 on padding), else it stays empty.
void build_graph(fa2_ctx *c, const fa2_graph_desc *g, float delta, std::vector<uint32_t> &off,
                 std::vector<int32_t> &col, std::vector<float> &wcol,
                 std::vector<float> &mass) {
    const uint32_t n = c->n;
    std::vector<uint32_t> deg(n, 0);
    for (uint64_t e = 0; e < g->num_edges; ++e) {
        deg[g->sources[e]]++;
        deg[g->targets[e]]++;
    }
    c->ref_of.resize(n);
    std::iota(c->ref_of.begin(), c->ref_of.end(), 0u);
    std::stable_sort(c->ref_of.begin(), c->ref_of.end(),
                     [&](uint32_t a, uint32_t b) { return deg[a] > deg[b]; });
    std::vector<uint32_t> int_of(n);
    for (uint32_t i = 0; i < n; ++i) int_of[c->ref_of[i]] = i;
    off.assign((size_t)n + 1, 0);
    mass.resize(n);
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t d = deg[c->ref_of[i]];
        off[i + 1] = off[i] + ((d + 3u) & ~3u);
        mass[i] = (float)d + 1.0f;  // ForceAtlas2::mass (src/RPForceAtlas2.cpp:74-77)
    }
    c->nnz_pad = off[n];
    col.assign(std::max<uint64_t>(c->nnz_pad, 4), 0);
    std::vector<uint32_t> fill(off.begin(), off.end() - 1);
    const bool weighted = g->weights && delta != 0.0f;
    if (!weighted) {
        wcol.clear();
        for (uint64_t e = 0; e < g->num_edges; ++e) {
            uint32_t a = int_of[g->sources[e]], b = int_of[g->targets[e]];
            col[fill[a]++] = (int32_t)b;
            col[fill[b]++] = (int32_t)a;
        }
        for (uint32_t i = 0; i < n; ++i) {
            std::sort(col.begin() + off[i], col.begin() + fill[i]);
            for (uint32_t q = fill[i]; q < off[i + 1]; ++q) col[q] = (int32_t)i;
        }
    } else {
        // (neighbour id, w^delta bits) pairs, sorted by id: ids are unique in a row
        std::vector<uint64_t> pair(col.size(), 0);
        for (uint64_t e = 0; e < g->num_edges; ++e) {
            uint32_t a = int_of[g->sources[e]], b = int_of[g->targets[e]];
            const float wd = (float)std::pow((double)g->weights[e], (double)delta);
            uint32_t bits;
            memcpy(&bits, &wd, 4);
            pair[fill[a]++] = (uint64_t)b << 32 | bits;
            pair[fill[b]++] = (uint64_t)a << 32 | bits;
        }
        wcol.assign(col.size(), 1.0f);
        for (uint32_t i = 0; i < n; ++i) {
            std::sort(pair.begin() + off[i], pair.begin() + fill[i]);
            for (uint32_t q = off[i]; q < fill[i]; ++q) {
                col[q] = (int32_t)(pair[q] >> 32);
                const uint32_t bits = (uint32_t)pair[q];
                memcpy(&wcol[q], &bits, 4);
            }
            for (uint32_t q = fill[i]; q < off[i + 1]; ++q) col[q] = (int32_t)i;
        }
    }
    // buckets: lanes per row from the number of 16-byte loads per row
    auto lanes_for = [](uint32_t q) -> int {
        if (q >= 512) return 256;
        if (q > 16) return 32;
        int l = 1;
        while (l < (int)q) l <<= 1;
        return l;
    };
    AttractPlan &P = c->plan;
    memset(&P, 0, sizeof(P));
    uint32_t r = 0;
    int blocks = 0;
    while (r < n && P.nbuckets < kMaxBuckets) {
        int lanes = lanes_for((off[r + 1] - off[r]) / 4);
        uint32_t r1 = r;
        while (r1 < n && lanes_for((off[r1 + 1] - off[r1]) / 4) == lanes) ++r1;
        AttractBucket &bk = P.b[P.nbuckets++];
        bk.row_begin = (int)r;
        bk.row_end = (int)r1;
        bk.lanes = lanes;
        bk.block_begin = blocks;
        int rows_per_block = lanes == 256 ? 1
                             : lanes == 32 ? 256 / 32
                                           : (256 / 32) * (32 / lanes) * kAttractBatch;
        blocks += (int)((r1 - r + rows_per_block - 1) / rows_per_block);
        r = r1;
    }
    P.nblocks = blocks;
}

// Enqueues one iteration.  full = false is the replay of a poisoned
// iteration: gravity, attraction and the bounding box were computed from the
// positions before the .99 scaling, as in the reference, and are kept.
void enqueue_iteration(fa2_ctx *c, bool full, bool perturb_first, bool timed) {
    const Buffers &b = c->b;
    cudaStream_t A = c->sA, B = c->sB;
    auto mark = [&](int slot, int end, cudaStream_t s) {
        if (timed)
            cudaEventRecordWithFlags(c->slot_events[slot * 2 + end], s, cudaEventRecordExternal);
    };
    const bool learn = c->learn_on;
    // the moment scan and per-cell second moments of the quadrupole walk
    const bool quad = c->kp.multipole >= 2;
    const bool side = full && c->overlap;  // stream B carries the attraction
    cudaMemsetAsync(c->scratch, 0, c->scratch_bytes, A);
    if (learn) cudaMemsetAsync(c->lb.corr, 0, ((size_t)c->n + 31) / 32 * sizeof(float2), A);
    if (full && !c->overlap) {
        mark(S_ATTRACT, 0, A);
        launch_attract(b, c->kp, c->plan, A);
        mark(S_ATTRACT, 1, A);
    } else if (full) {
        cudaEventRecord(c->evFork, A);
        cudaStreamWaitEvent(B, c->evFork, 0);
        mark(S_ATTRACT, 0, B);
        launch_attract(b, c->kp, c->plan, B);
        mark(S_ATTRACT, 1, B);
        if (!quad) cudaEventRecord(c->evJoin, B);
    }
    if (perturb_first) launch_runs(b, 1, c->nsm, A);
    mark(S_KEYS, 0, A);
    launch_keys(b, c->nsm, A);
    mark(S_KEYS, 1, A);
    mark(S_SORT, 0, A);
    launch_sort(b, A);
    launch_fix_low(b, c->nsm, A);
    mark(S_SORT, 1, A);
    mark(S_COUNT, 0, A);
    launch_tree_count(b, quad, A);
    mark(S_COUNT, 1, A);
    // The tree count leaves the sorted bodies' grid offsets and masses for the
    // moment scan; with stream B in use the scan runs there, beside the emit.
    if (quad) {
        cudaStream_t M = side ? B : A;
        if (side) {
            cudaEventRecord(c->evCounted, A);
            cudaStreamWaitEvent(B, c->evCounted, 0);
        }
        mark(S_MOM, 0, M);
        launch_moments(b, M);
        mark(S_MOM, 1, M);
        if (side) cudaEventRecord(c->evJoin, B);
    }
    mark(S_EMIT, 0, A);
    launch_emit(b, c->nsm, A);
    mark(S_EMIT, 1, A);
    if (learn) {
        // the cells' second moments (a feature of the pairs), beside the walk
        // on stream B when it is in use; the MLP waits for them
        cudaStream_t M = side ? B : A;
        if (side) {
            cudaEventRecord(c->evEmitted, A);
            cudaStreamWaitEvent(B, c->evEmitted, 0);
        }
        // timed in the moments slot, which the monopole walk leaves free
        if (!quad) mark(S_MOM, 0, M);
        launch_cell_a2(b, c->lb, c->nsm, M);
        if (!quad) mark(S_MOM, 1, M);
        if (side) cudaEventRecord(c->evA2, B);
    }
    if (side) cudaStreamWaitEvent(A, c->evJoin, 0);
    if (quad) {
        mark(S_QUAD, 0, A);
        launch_quad_cells(b, c->nsm, A);
        mark(S_QUAD, 1, A);
    }
    if (c->kp.overlap) launch_sorted_sizes(b, A);
    mark(S_TRAV, 0, A);
    if (learn)
        launch_traverse_learn(b, c->kp, c->lb, c->trav_blocks, A);
    else
        launch_traverse(b, c->kp, c->trav_blocks, A);
    mark(S_TRAV, 1, A);
    if (learn) {
        if (side) cudaStreamWaitEvent(A, c->evA2, 0);
        mark(S_LEARN, 0, A);
        launch_learn_mlp(b, c->kp, c->lb, c->nsm, A);
        launch_learn_tail(b, c->kp, c->lb, c->nsm, A);
        mark(S_LEARN, 1, A);
    }
    mark(S_DISP, 0, A);
    launch_displace(b, c->nsm, A);
    mark(S_DISP, 1, A);
}

int capture(fa2_ctx *c, bool timed, cudaGraphExec_t *out) {
    cudaGraph_t graph = nullptr;
    CK(cudaStreamBeginCapture(c->sA, cudaStreamCaptureModeThreadLocal));
    enqueue_iteration(c, true, false, timed);
    cudaError_t e = cudaStreamEndCapture(c->sA, &graph);
    if (e != cudaSuccess) return cuda_status(e);
    e = cudaGraphInstantiate(out, graph, cudaGraphInstantiateFlagUseNodePriority);
    if (e == cudaSuccess && timed) {
        size_t nn = 0;
        cudaGraphGetNodes(graph, nullptr, &nn);
        std::vector<cudaGraphNode_t> nodes(nn);
        cudaGraphGetNodes(graph, nodes.data(), &nn);
        c->timed_nodes.assign(kNumSlots * 2, nullptr);
        for (cudaGraphNode_t nd : nodes) {
            cudaGraphNodeType t;
            cudaGraphNodeGetType(nd, &t);
            if (t != cudaGraphNodeTypeEventRecord) continue;
            cudaEvent_t ev;
            cudaGraphEventRecordNodeGetEvent(nd, &ev);
            for (int s = 0; s < kNumSlots * 2; ++s)
                if (c->slot_events[s] == ev) c->timed_nodes[s] = nd;
        }
    }
    if (timed)
        c->graph_timed = graph;
    else
        cudaGraphDestroy(graph);
    return cuda_status(e);
}

// The guard checks only an approximation other than the reference's.
bool guard_active(const fa2_ctx *c) {
    return c->guard_every > 0 && (c->kp.multipole >= 2 || c->kp.itolsq != 1.0f || c->learn_on);
}

// One check of the accuracy guard on the last iteration's tree: relative RMSE
// of the applied repulsion and of the plain walk against the FP64 sum over
// the sampled bodies; the plain walk takes over when it is the more accurate.
int guard_check(fa2_ctx *c) {
    const int ns = c->guard_samples;
    launch_guard(c->b, c->kp, ns, c->guard_exact, c->guard_plain, c->guard_cur, c->guard_part,
                 c->sA);
    CK(cudaGetLastError());
    std::vector<double2> ex((size_t)ns);
    std::vector<float2> pl((size_t)ns), cu((size_t)ns);
    CK(cudaMemcpyAsync(ex.data(), c->guard_exact, ex.size() * sizeof(double2),
                       cudaMemcpyDeviceToHost, c->sA));
    CK(cudaMemcpyAsync(pl.data(), c->guard_plain, pl.size() * sizeof(float2),
                       cudaMemcpyDeviceToHost, c->sA));
    CK(cudaMemcpyAsync(cu.data(), c->guard_cur, cu.size() * sizeof(float2),
                       cudaMemcpyDeviceToHost, c->sA));
    CK(cudaStreamSynchronize(c->sA));
    double e_cur = 0.0, e_plain = 0.0, norm = 0.0;
    for (int s = 0; s < ns; ++s) {
        const double ax = cu[s].x - ex[s].x, ay = cu[s].y - ex[s].y;
        const double bx = pl[s].x - ex[s].x, by = pl[s].y - ex[s].y;
        e_cur += ax * ax + ay * ay;
        e_plain += bx * bx + by * by;
        norm += ex[s].x * ex[s].x + ex[s].y * ex[s].y;
    }
    if (!(norm > 0.0)) return FA2_OK;  // nothing to compare against
    c->guard_err_cur = std::sqrt(e_cur / norm);
    c->guard_err_plain = std::sqrt(e_plain / norm);
    c->guard_checks += 1;
    if (c->guard_err_cur > c->guard_err_plain) {
        // back to the reference's walk: theta 1, cells as point masses, no
        // learned correction
        c->kp.itolsq = 1.0f;
        c->kp.multipole = 1;
        c->learn_on = false;
        c->prm.theta = 1.0f;
        c->prm.multipole = 1;
        c->guard_fallbacks += 1;
        drop_graphs(c);
    }
    return FA2_OK;
}

int read_state(fa2_ctx *c, DevState *st) {
    CK(cudaMemcpyAsync(st, c->b.st, sizeof(DevState), cudaMemcpyDeviceToHost, c->sA));
    CK(cudaStreamSynchronize(c->sA));
    return FA2_OK;
}

// Replays a poisoned iteration until no coincident bodies remain.
int resolve_poison(fa2_ctx *c, DevState *st) {
    int rounds = 0;
    while (st->poison) {
        if (++rounds > kMaxReplayRounds) return FA2_ERR_DEVICE_LIMIT;
        // A run of keys equal in the sorted digits was too long for
        // k_fix_low: the iteration again, sorted on every digit.  Otherwise
        // coincident bodies: the iteration again after the .99 scaling.
        const bool resort = st->resort != 0;
        if (resort) {
            c->b.sort_first = 0;
            drop_graphs(c);
            CK(cudaMemsetAsync(&c->b.st->resort, 0, sizeof(int), c->sA));
        }
        CK(cudaMemsetAsync(&c->b.st->poison, 0, sizeof(int), c->sA));
        enqueue_iteration(c, false, !resort, false);
        CK(cudaGetLastError());
        int s = read_state(c, st);
        if (s) return s;
        if (st->err) return FA2_ERR_DEVICE_LIMIT;
    }
    c->last_perturb_rounds = rounds;
    return FA2_OK;
}

// After a tree no deeper than kShallowLevel (kMidLevel) the next sorts skip
// their two lowest digits (their lowest one); k_fix_low keeps the order
// exact.  The choice is part of the captured graphs, which are dropped when
// it changes.
void choose_sort_passes(fa2_ctx *c, const DevState &st) {
    const int l = st.max_level;
    const int first = l <= 0 ? 0 : (l <= kShallowLevel ? 2 : (l <= kMidLevel ? 1 : 0));
    if (first == c->b.sort_first) return;
    c->b.sort_first = first;
    drop_graphs(c);
}

// Runs n iterations; with `timed`, kernel_sum accumulates per-slot device ms.
int run_steps(fa2_ctx *c, int32_t n_iters, bool timed, std::vector<double> *kernel_sum,
              std::vector<int> *kernel_cnt) {
    if (n_iters <= 0 || c->n == 0) return FA2_OK;
    cudaGraphExec_t *exec = timed ? &c->exec_timed : &c->exec;
    DevState st;
    int s = read_state(c, &st);
    if (s) return s;
    int done = 0;
    c->last_perturb_rounds = 0;
    while (done < n_iters) {
        choose_sort_passes(c, st);
        // (re)captured here: a guard fallback drops the graphs
        if (!*exec) {
            s = capture(c, timed, exec);
            if (s) return s;
        }
        const bool guard = guard_active(c);
        const int before = st.iters_done;
        int chunk = n_iters - done;
        if (guard) chunk = std::min(chunk, std::max(c->guard_left, 1));
        if (timed) {
            size_t need = (size_t)chunk * kNumSlots * 2;
            while (c->event_pool.size() < need) {
                cudaEvent_t e;
                CK(cudaEventCreate(&e));
                c->event_pool.push_back(e);
            }
        }
        for (int it = 0; it < chunk; ++it) {
            if (timed)
                for (int q = 0; q < kNumSlots * 2; ++q)
                    if (c->timed_nodes[q])
                        CK(cudaGraphExecEventRecordNodeSetEvent(
                            *exec, c->timed_nodes[q], c->event_pool[(size_t)it * kNumSlots * 2 + q]));
            CK(cudaGraphLaunch(*exec, c->sA));
        }
        s = read_state(c, &st);
        if (s) return s;
        if (st.err) return FA2_ERR_DEVICE_LIMIT;
        int completed = st.iters_done - before;
        if (timed && kernel_sum) {
            for (int it = 0; it < completed; ++it)
                for (int q = 0; q < kNumSlots; ++q) {
                    if (!c->timed_nodes[2 * q] || !c->timed_nodes[2 * q + 1]) continue;
                    float ms = 0.0f;
                    size_t base = (size_t)it * kNumSlots * 2;
                    if (cudaEventElapsedTime(&ms, c->event_pool[base + 2 * q],
                                             c->event_pool[base + 2 * q + 1]) == cudaSuccess) {
                        (*kernel_sum)[q] += ms;
                        (*kernel_cnt)[q] += 1;
                    }
                }
        }
        done += completed;
        if (st.poison) {
            s = resolve_poison(c, &st);
            if (s) return s;
            done += 1;  // the replayed iteration completed
            completed += 1;
        }
        if (guard) {
            c->guard_left -= completed;
            if (c->guard_left <= 0) {
                c->guard_left = c->guard_every;
                s = guard_check(c);
                if (s) return s;
            }
        }
    }
    return FA2_OK;
}


// ------------------------------------------------ learned correction --

// Round to the nearest BF16 (ties to even), as bits and as a float.
uint16_t bf16_bits(float x) {
    uint32_t u;
    memcpy(&u, &x, 4);
    if ((u & 0x7F800000u) == 0x7F800000u && (u & 0x007FFFFFu)) return (uint16_t)((u >> 16) | 0x40u);
    u += 0x7FFFu + ((u >> 16) & 1u);
    return (uint16_t)(u >> 16);
}

float bf16_value(float x) {
    const uint32_t u = (uint32_t)bf16_bits(x) << 16;
    float f;
    memcpy(&f, &u, 4);
    return f;
}

bool mlp_is_finite(const fa2_mlp &m) {
    const float *p = reinterpret_cast<const float *>(&m);
    for (size_t i = 0; i < sizeof(fa2_mlp) / sizeof(float); ++i)
        if (!std::isfinite(p[i])) return false;
    return true;
}

// The FP32 parameters as the kernels read them (MlpDevice): W1, W2 and W3 in
// BF16 in the tensor cores' operand layout, b1 and b2 as BF16 pairs (value and
// rest) in W1's and W2's extra K columns, W3 padded to 16 rows, b3 as given.
void mlp_to_device(const fa2_mlp &m, MlpDevice &d) {
    memset(&d, 0, sizeof(d));
    for (int j = 0; j < kLearnHidden; ++j) {
        for (int k = 0; k < kLearnInPad; ++k) {
            uint16_t v = 0;
            if (k < kLearnIn) v = bf16_bits(m.w1[j * kLearnIn + k]);
            // b1 = hi + lo in BF16, against the features' two columns of ones
            if (k == kBiasColHi) v = bf16_bits(m.b1[j]);
            if (k == kBiasColLo) v = bf16_bits(m.b1[j] - bf16_value(m.b1[j]));
            d.w1[operand_offset(j, k, kLearnInPad / 8) / 2] = v;
        }
        for (int k = 0; k < kLearnHidPad; ++k) {
            uint16_t v = 0;
            if (k < kLearnHidden) v = bf16_bits(m.w2[j * kLearnHidden + k]);
            // b2 = hi + lo against the hidden tile's two columns of ones
            if (k == kBias2ColHi) v = bf16_bits(m.b2[j]);
            if (k == kBias2ColLo) v = bf16_bits(m.b2[j] - bf16_value(m.b2[j]));
            d.w2[operand_offset(j, k, kLearnHidPad / 8) / 2] = v;
        }
        for (int o = 0; o < kLearnOut; ++o)
            d.w3[operand_offset(o, j, kLearnHidden / 8) / 2] = bf16_bits(m.w3[o * kLearnHidden + j]);
    }
    d.b3[0] = m.b3[0];
    d.b3[1] = m.b3[1];
}

// nn.Linear's default initialisation: U(-1/sqrt(fan_in), 1/sqrt(fan_in)).
void mlp_default_init(fa2_mlp *m, uint32_t seed) {
    std::mt19937 rng(seed);
    auto fill = [&](float *p, int count, int fan_in) {
        const float bound = 1.0f / std::sqrt((float)fan_in);
        std::uniform_real_distribution<float> u(-bound, bound);
        for (int i = 0; i < count; ++i) p[i] = u(rng);
    };
    fill(m->w1, kLearnHidden * kLearnIn, kLearnIn);
    fill(m->b1, kLearnHidden, kLearnIn);
    fill(m->w2, kLearnHidden * kLearnHidden, kLearnHidden);
    fill(m->b2, kLearnHidden, kLearnHidden);
    fill(m->w3, kLearnOut * kLearnHidden, kLearnHidden);
    fill(m->b3, kLearnOut, kLearnHidden);
}

// Makes `device` current after checking it is an sm_100 part.
int use_device(int device, int *nsm) {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
        return FA2_ERR_NO_DEVICE;
    cudaDeviceProp dp;
    if (cudaGetDeviceProperties(&dp, device) != cudaSuccess || dp.major < 10)
        return FA2_ERR_NO_DEVICE;
    if (cudaSetDevice(device) != cudaSuccess) return FA2_ERR_CUDA;
    *nsm = dp.multiProcessorCount;
    return FA2_OK;
}

// Device buffers and a stream for the length of one call.
struct DeviceScratch {
    std::vector<void *> ptrs;
    cudaStream_t stream = nullptr;
    DeviceScratch() { cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking); }
    ~DeviceScratch() {
        if (stream) cudaStreamSynchronize(stream);
        for (void *p : ptrs) cudaFree(p);
        if (stream) cudaStreamDestroy(stream);
    }
    template <typename T>
    int get(T **p, size_t count) {
        void *q = nullptr;
        const cudaError_t e = cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T));
        if (e != cudaSuccess) return cuda_status(e);
        ptrs.push_back(q);
        *p = (T *)q;
        return stream ? FA2_OK : FA2_ERR_CUDA;
    }
};

}  // namespace

struct fa2_learn_set {
    int device = 0;
    int64_t cap = 0, size = 0;
    float *feat = nullptr;  // cap x 12
    float2 *tgt = nullptr;
    float *w = nullptr;
    cudaStream_t stream = nullptr;
    // one collect's samples before they are put in order
    int64_t st_cap = 0;
    float *st_feat = nullptr;
    float2 *st_tgt = nullptr;
    float *st_w = nullptr;
    uint64_t *st_key = nullptr;
    unsigned long long *st_count = nullptr;
};

namespace {

int set_staging(fa2_learn_set *set, int64_t need) {
    if (set->st_cap >= need && set->st_count) return FA2_OK;
    cudaFree(set->st_feat);
    cudaFree(set->st_tgt);
    cudaFree(set->st_w);
    cudaFree(set->st_key);
    cudaFree(set->st_count);
    set->st_feat = nullptr;
    set->st_tgt = nullptr;
    set->st_w = nullptr;
    set->st_key = nullptr;
    set->st_count = nullptr;
    set->st_cap = 0;
    const size_t k = (size_t)need;
    CK(cudaMalloc(&set->st_feat, k * kLearnIn * 4));
    CK(cudaMalloc(&set->st_tgt, k * 8));
    CK(cudaMalloc(&set->st_w, k * 4));
    CK(cudaMalloc(&set->st_key, k * 8));
    CK(cudaMalloc(&set->st_count, sizeof(unsigned long long)));
    set->st_cap = need;
    return FA2_OK;
}

}  // namespace

extern "C" {

void fa2_default_params(fa2_params *p) {
    if (!p) return;
    p->use_barneshut = 1;
    p->strong_gravity = 0;
    p->gravity = 1.0f;
    p->scale = 1.0f;
    p->theta = 1.0f;
    p->epssq = 0.05 * 0.05;
    p->jitter_tolerance = 1.0f;
    p->k_s_max = 10.0f;
    p->device = 0;
    p->linlog = 0;
    p->multipole = 1;
    p->delta = 0.0f;
}

fa2_ctx *fa2_create(const fa2_graph_desc *g, const fa2_params *prm, int *status) {
    int dummy;
    if (!status) status = &dummy;
    *status = FA2_ERR_INVALID_ARGUMENT;
    if (!g || !prm) return nullptr;
    if (g->num_edges && (!g->sources || !g->targets)) return nullptr;
    if (!prm->use_barneshut) {
        *status = FA2_ERR_UNSUPPORTED;
        return nullptr;
    }
    if (!(prm->theta > 0.0f)) return nullptr;
    for (uint64_t e = 0; e < g->num_edges; ++e)
        if (g->sources[e] >= g->num_nodes || g->targets[e] >= g->num_nodes ||
            g->sources[e] == g->targets[e])
            return nullptr;
    // edge weights: finite and positive, and w^delta finite and positive
    if (!std::isfinite(prm->delta)) return nullptr;
    if (g->weights && prm->delta != 0.0f)
        for (uint64_t e = 0; e < g->num_edges; ++e) {
            const float w = g->weights[e];
            if (!(w > 0.0f) || !std::isfinite(w)) return nullptr;
            const double wd = std::pow((double)w, (double)prm->delta);
            if (!(wd >= (double)FLT_MIN && wd <= (double)FLT_MAX)) return nullptr;
        }
    if ((uint64_t)g->num_nodes * 2 + 2 * g->num_edges + 3ull * g->num_nodes >= (1ull << 32) ||
        g->num_nodes >= (1u << 25)) {
        *status = FA2_ERR_TOO_LARGE;
        return nullptr;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= prm->device || prm->device < 0) {
        *status = FA2_ERR_NO_DEVICE;
        return nullptr;
    }
    cudaDeviceProp dp;
    if (cudaGetDeviceProperties(&dp, prm->device) != cudaSuccess || dp.major < 10) {
        *status = FA2_ERR_NO_DEVICE;
        return nullptr;
    }
    if (cudaSetDevice(prm->device) != cudaSuccess) {
        *status = FA2_ERR_CUDA;
        return nullptr;
    }
    fa2_ctx *c = new fa2_ctx();
    c->device = prm->device;
    c->nsm = dp.multiProcessorCount;
    c->n = g->num_nodes;
    c->m = g->num_edges;
    c->prm = *prm;
    c->kp.k_r = prm->scale;
    c->kp.k_g = prm->gravity;
    c->kp.itolsq = 1.0f / (prm->theta * prm->theta);  // src/RPForceAtlas2.cpp:47
    c->kp.epssq = prm->epssq;
    c->kp.strong_gravity = prm->strong_gravity;
    c->kp.linlog = prm->linlog != 0;
    c->kp.multipole = prm->multipole >= 2 ? 2 : 1;

    std::vector<uint32_t> off;
    std::vector<int32_t> col;
    std::vector<float> wcol, mass;
    build_graph(c, g, prm->delta, off, col, wcol, mass);

    auto fail = [&](int s) {
        *status = s;
        free_all(c);
        delete c;
        return (fa2_ctx *)nullptr;
    };
    const uint32_t n = c->n;
    Buffers &b = c->b;
    b.n = (int)n;
    uint64_t cap = std::min<uint64_t>(33ull * n + 64, kMaxTreeNodes);
    b.capacity = (uint32_t)cap;
    uint32_t *d_off = nullptr, *d_ref = nullptr;
    int4 *d_col = nullptr;
    float4 *d_w = nullptr;
    int s = FA2_OK;
    if ((s = dalloc(c, &b.pos, n)) || (s = dalloc(c, &b.fprev, n)) || (s = dalloc(c, &b.f, n)) ||
        (s = dalloc(c, &b.fag, n)) || (s = dalloc(c, &b.mass, n)) ||
        (s = dalloc(c, &d_off, (size_t)n + 1)) || (s = dalloc(c, &d_col, col.size() / 4)) ||
        (s = dalloc(c, &d_ref, n)) || (s = dalloc(c, &b.keys[0], n)) ||
        (s = dalloc(c, &b.keys[1], n)) || (s = dalloc(c, &b.vals[0], n)) ||
        (s = dalloc(c, &b.vals[1], n)) || (s = dalloc(c, &b.lcp, n)) ||
        (s = dalloc(c, &b.group, n)) || (s = dalloc(c, &b.body_node, n)) ||
        (s = dalloc(c, &b.nodes, cap + 1)) ||  // + one spare slot
        (s = dalloc(c, &b.owner, cap)) ||
        (s = dalloc(c, &b.pm, (size_t)n + 1)) || (s = dalloc(c, &b.pxy, 2 * ((size_t)n + 1))) ||
        (s = dalloc(c, &b.lookback, (size_t)count_tiles((int)n))) ||
        (s = dalloc(c, &b.warp_partial, (n + 31) / 32)) ||
        (s = dalloc(c, &b.st, 1)) || (s = dalloc(c, &c->stage_xy, n)) ||
        (s = dalloc(c, &c->stage_ids, n)))
        return fail(s);
    if (c->kp.multipole >= 2 && (s = ensure_quad_buffers(c))) return fail(s);
    c->bbox_blocks = c->nsm * 2;
    // partial boxes of k_bbox (bbox_blocks) and of k_displace (up to 4 per SM)
    if ((s = dalloc(c, &b.bbox_partial, (size_t)c->nsm * 4))) return fail(s);
    if (!wcol.empty() && (s = dalloc(c, &d_w, wcol.size() / 4))) return fail(s);
    c->kp.nsm = c->nsm;
    b.csr_off = d_off;
    b.csr_col4 = d_col;
    b.csr_w4 = d_w;
    b.ref_of = d_ref;
    // one memset clears counters, histograms, per-tile digit counts and the
    // tree-count look-back flags
    b.sort_rounds = sort_rounds((int)n, c->nsm);
    const size_t sort_counts = (size_t)8 * sort_tiles_max((int)n) * 256;
    const size_t count_status = (size_t)count_tiles((int)n);
    const size_t mom_status = (size_t)mom_tiles((int)n);
    c->scratch_bytes = sizeof(IterCounters) + 4 * (sort_counts + count_status + mom_status);
    char *scr = nullptr;
    if ((s = dalloc(c, &scr, c->scratch_bytes))) return fail(s);
    c->scratch = scr;
    b.ctr = (IterCounters *)scr;
    b.sort_counts = (uint32_t *)(scr + sizeof(IterCounters));
    b.count_status = b.sort_counts + sort_counts;
    b.mom_status = b.count_status + count_status;

    // The tree chain (stream A) is the critical path; the attraction (stream B)
    // only has to finish before the traversal.  With A at the higher priority
    // the block scheduler starts A's blocks first and fills the rest of the
    // SMs with attraction blocks, instead of holding the chain behind them.
    int prio_low = 0, prio_high = 0;
    cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high);
    if (cudaStreamCreateWithPriority(&c->sA, cudaStreamNonBlocking, prio_high) != cudaSuccess ||
        cudaStreamCreateWithPriority(&c->sB, cudaStreamNonBlocking, prio_low) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->evFork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->evJoin, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->evCounted, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->evEmitted, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->evA2, cudaEventDisableTiming) != cudaSuccess ||
        cudaMallocHost(&c->h_state, sizeof(DevState)) != cudaSuccess ||
        cudaMallocHost(&c->h_iters, sizeof(int)) != cudaSuccess)
        return fail(FA2_ERR_CUDA);
    c->slot_events.resize(kNumSlots * 2);
    for (auto &e : c->slot_events)
        if (cudaEventCreate(&e) != cudaSuccess) return fail(FA2_ERR_CUDA);
    sort_set_smem_attr();
    c->trav_blocks = c->nsm * traverse_blocks_per_sm();

    cudaStream_t A = c->sA;
    if (cudaMemcpyAsync(d_off, off.data(), off.size() * 4, cudaMemcpyHostToDevice, A) ||
        cudaMemcpyAsync(d_col, col.data(), col.size() * 4, cudaMemcpyHostToDevice, A) ||
        (d_w && cudaMemcpyAsync(d_w, wcol.data(), wcol.size() * 4, cudaMemcpyHostToDevice, A)) ||
        cudaMemcpyAsync(d_ref, c->ref_of.data(), (size_t)n * 4, cudaMemcpyHostToDevice, A) ||
        cudaMemcpyAsync(b.mass, mass.data(), (size_t)n * 4, cudaMemcpyHostToDevice, A) ||
        cudaMemsetAsync(b.pos, 0, (size_t)n * 8, A) || cudaMemsetAsync(b.fprev, 0, (size_t)n * 8, A) ||
        cudaMemsetAsync(b.f, 0, (size_t)n * 8, A) || cudaMemsetAsync(b.fag, 0, (size_t)n * 8, A) ||
        cudaMemsetAsync(b.st, 0, sizeof(DevState), A))
        return fail(FA2_ERR_CUDA);
    DevState st0;
    memset(&st0, 0, sizeof(st0));
    st0.global_speed = 1.0f;      // src/RPFA2Kernels.cu:30
    st0.speed_efficiency = 1.0f;  // :31
    st0.jitter_tolerance = prm->jitter_tolerance;
    st0.k_s_max = prm->k_s_max;
    if (cudaMemcpyAsync(b.st, &st0, sizeof(st0), cudaMemcpyHostToDevice, A) ||
        cudaStreamSynchronize(A))
        return fail(FA2_ERR_CUDA);
    *status = FA2_OK;
    return c;
}

void fa2_destroy(fa2_ctx *c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->sA) cudaStreamSynchronize(c->sA);
    if (c->sB) cudaStreamSynchronize(c->sB);
    free_all(c);
    delete c;
}

int fa2_set_positions(fa2_ctx *c, const float *xy) {
    if (!c || (!xy && c->n)) return FA2_ERR_INVALID_ARGUMENT;
    CK(cudaSetDevice(c->device));
    if (c->n == 0) return FA2_OK;
    const size_t bytes = (size_t)c->n * 8;
    CK(cudaMemcpyAsync(c->stage_xy, xy, bytes, cudaMemcpyHostToDevice, c->sA));
    launch_scatter_xy((int)c->n, c->b.ref_of, c->stage_xy, c->b.pos, c->sA);
    // the root cell of the next tree comes from these positions; device
    // errors of earlier positions are cleared (k_bbox flags non-finite ones)
    CK(cudaMemsetAsync(c->scratch, 0, c->scratch_bytes, c->sA));
    CK(cudaMemsetAsync(&c->b.st->err, 0, sizeof(int), c->sA));
    launch_bbox(c->b, c->bbox_blocks, c->sA);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(c->sA));
    return FA2_OK;
}

int fa2_get_positions(fa2_ctx *c, float *xy) {
    if (!c || (!xy && c->n)) return FA2_ERR_INVALID_ARGUMENT;
    CK(cudaSetDevice(c->device));
    if (c->n == 0) return FA2_OK;
    launch_gather_xy((int)c->n, c->b.ref_of, c->b.pos, c->stage_xy, c->sA);
    CK(cudaMemcpyAsync(xy, c->stage_xy, (size_t)c->n * 8, cudaMemcpyDeviceToHost, c->sA));
    CK(cudaStreamSynchronize(c->sA));
    return FA2_OK;
}

int fa2_step(fa2_ctx *c, int32_t n_iters) {
    if (!c || n_iters < 0) return FA2_ERR_INVALID_ARGUMENT;
    CK(cudaSetDevice(c->device));
    return run_steps(c, n_iters, false, nullptr, nullptr);
}

int fa2_step_host(fa2_ctx *c, const float *xy_in, int32_t n_iters, float *xy_out) {
    if (!c || n_iters < 0) return FA2_ERR_INVALID_ARGUMENT;
    CK(cudaSetDevice(c->device));
    if (c->n == 0) return FA2_OK;
    int s = FA2_OK;
    if (guard_active(c)) {
        // the guard's checks sit between iterations: the separate calls
        if (xy_in && (s = fa2_set_positions(c, xy_in))) return s;
        if ((s = run_steps(c, n_iters, false, nullptr, nullptr))) return s;
        return xy_out ? fa2_get_positions(c, xy_out) : FA2_OK;
    }
    if (n_iters > 0 && !c->exec && (s = capture(c, false, &c->exec))) return s;
    cudaStream_t A = c->sA;
    const size_t bytes = (size_t)c->n * 8;
    if (xy_in) {
        // fa2_set_positions without its synchronisation
        CK(cudaMemcpyAsync(c->stage_xy, xy_in, bytes, cudaMemcpyHostToDevice, A));
        launch_scatter_xy((int)c->n, c->b.ref_of, c->stage_xy, c->b.pos, A);
        CK(cudaMemsetAsync(c->scratch, 0, c->scratch_bytes, A));
        CK(cudaMemsetAsync(&c->b.st->err, 0, sizeof(int), A));
        launch_bbox(c->b, c->bbox_blocks, A);
    }
    CK(cudaMemcpyAsync(c->h_iters, &c->b.st->iters_done, sizeof(int), cudaMemcpyDeviceToHost, A));
    c->last_perturb_rounds = 0;
    for (int it = 0; it < n_iters; ++it) CK(cudaGraphLaunch(c->exec, A));
    CK(cudaMemcpyAsync(c->h_state, c->b.st, sizeof(DevState), cudaMemcpyDeviceToHost, A));
    if (xy_out) {
        launch_gather_xy((int)c->n, c->b.ref_of, c->b.pos, c->stage_xy, A);
        CK(cudaMemcpyAsync(xy_out, c->stage_xy, bytes, cudaMemcpyDeviceToHost, A));
    }
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(A));
    DevState st = *c->h_state;
    if (st.err) return FA2_ERR_DEVICE_LIMIT;
    int completed = st.iters_done - *c->h_iters;
    if (completed == n_iters && !st.poison) {
        choose_sort_passes(c, st);
        return FA2_OK;
    }
    // An iteration was replayed (coincident bodies, or a sort that needs all
    // its digits): the iterations after it did nothing.  The rest as
    // fa2_step does it, then the positions again.
    if (st.poison) {
        if ((s = resolve_poison(c, &st))) return s;
        completed += 1;
    }
    if (completed < n_iters && (s = run_steps(c, n_iters - completed, false, nullptr, nullptr)))
        return s;
    return xy_out ? fa2_get_positions(c, xy_out) : FA2_OK;
}

int fa2_step_timed(fa2_ctx *c, int32_t n_iters, float *ms_total, float *kernel_ms,
                   int32_t n_kernels) {
    if (!c || n_iters < 0 || !ms_total) return FA2_ERR_INVALID_ARGUMENT;
    CK(cudaSetDevice(c->device));
    cudaEvent_t t0, t1;
    CK(cudaEventCreate(&t0));
    CK(cudaEventCreate(&t1));
    std::vector<double> sum(kNumSlots, 0.0);
    std::vector<int> cnt(kNumSlots, 0);
    const bool per_kernel = kernel_ms && n_kernels > 0;
    cudaEventRecord(t0, c->sA);
    int s = per_kernel ? run_steps(c, n_iters, true, &sum, &cnt)
                       : run_steps(c, n_iters, false, nullptr, nullptr);
    cudaEventRecord(t1, c->sA);
    cudaEventSynchronize(t1);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, t0, t1);
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    *ms_total = ms;
    if (per_kernel)
        for (int q = 0; q < n_kernels && q < kNumSlots; ++q)
            kernel_ms[q] = cnt[q] ? (float)(sum[q] / cnt[q]) : 0.0f;
    return s;
}

const char *fa2_kernel_name(int32_t i) { return (i >= 0 && i < kNumSlots) ? kSlotNames[i] : nullptr; }

int fa2_get_stats(fa2_ctx *c, fa2_stats *out) {
    if (!c || !out) return FA2_ERR_INVALID_ARGUMENT;
    CK(cudaSetDevice(c->device));
    DevState st;
    memset(&st, 0, sizeof(st));
    if (c->n) {
        // interaction and visit counts: one counting walk over the last tree
        CK(cudaMemsetAsync(&c->b.st->interactions, 0, 2 * sizeof(unsigned long long), c->sA));
        launch_count_interactions(c->b, c->kp, c->trav_blocks, c->sA);
        CK(cudaGetLastError());
        int s = read_state(c, &st);
        if (s) return s;
    }
    memset(out, 0, sizeof(*out));
    out->num_bodies = c->n;
    out->tree_nodes = st.tree_nodes;
    out->tree_cells = st.tree_nodes >= c->n ? st.tree_nodes - c->n : 0;
    out->max_level = st.max_level;
    out->perturb_rounds = c->last_perturb_rounds;
    out->device_error = st.err;
    out->nnz_padded = c->nnz_pad;
    out->global_speed = st.global_speed;
    out->speed_efficiency = st.speed_efficiency;
    out->radius = st.radius;
    out->root_x = st.rootx;
    out->root_y = st.rooty;
    out->interactions = st.interactions;
    out->visits = st.visits;
    out->sort_passes = 8 - c->b.sort_first;
    if (c->learn_on && c->n) {
        unsigned counts[kPairSegments];
        CK(cudaMemcpyAsync(counts, c->b.ctr->pair_count, sizeof(counts), cudaMemcpyDeviceToHost,
                           c->sA));
        CK(cudaStreamSynchronize(c->sA));
        for (int q = 0; q < kPairSegments; ++q)
            out->learned_pairs += std::min(counts[q], c->lb.seg_cap);
    }
    return FA2_OK;
}

int fa2_get_forces(fa2_ctx *c, float *f_total, float *f_attr_grav) {
    if (!c) return FA2_ERR_INVALID_ARGUMENT;
    CK(cudaSetDevice(c->device));
    if (c->n == 0) return FA2_OK;
    float *outs[2] = {f_total, f_attr_grav};
    float2 *srcs[2] = {c->b.f, c->b.fag};
    for (int q = 0; q < 2; ++q) {
        if (!outs[q]) continue;
        launch_gather_xy((int)c->n, c->b.ref_of, srcs[q], c->stage_xy, c->sA);
        CK(cudaMemcpyAsync(outs[q], c->stage_xy, (size_t)c->n * 8, cudaMemcpyDeviceToHost, c->sA));
        CK(cudaStreamSynchronize(c->sA));
    }
    return FA2_OK;
}

int fa2_get_sort_order(fa2_ctx *c, uint32_t *order) {
    if (!c || (!order && c->n)) return FA2_ERR_INVALID_ARGUMENT;
    CK(cudaSetDevice(c->device));
    if (c->n == 0) return FA2_OK;
    launch_sorted_ref_ids((int)c->n, c->b.ref_of, c->b.vals[0], c->stage_ids, c->sA);
    CK(cudaMemcpyAsync(order, c->stage_ids, (size_t)c->n * 4, cudaMemcpyDeviceToHost, c->sA));
    CK(cudaStreamSynchronize(c->sA));
    return FA2_OK;
}

int fa2_set_speed_state(fa2_ctx *c, float global_speed, float speed_efficiency,
                        const float *f_prev) {
    if (!c) return FA2_ERR_INVALID_ARGUMENT;
    CK(cudaSetDevice(c->device));
    DevState st;
    int s = read_state(c, &st);
    if (s) return s;
    st.global_speed = global_speed;
    st.speed_efficiency = speed_efficiency;
    CK(cudaMemcpyAsync(c->b.st, &st, sizeof(st), cudaMemcpyHostToDevice, c->sA));
    if (c->n) {
        if (f_prev) {
            CK(cudaMemcpyAsync(c->stage_xy, f_prev, (size_t)c->n * 8, cudaMemcpyHostToDevice, c->sA));
            launch_scatter_xy((int)c->n, c->b.ref_of, c->stage_xy, c->b.fprev, c->sA);
        } else {
            CK(cudaMemsetAsync(c->b.fprev, 0, (size_t)c->n * 8, c->sA));
        }
    }
    CK(cudaStreamSynchronize(c->sA));
    return FA2_OK;
}

int fa2_get_speed_state(fa2_ctx *c, float *global_speed, float *speed_efficiency,
                        float *f_prev) {
    if (!c) return FA2_ERR_INVALID_ARGUMENT;
    CK(cudaSetDevice(c->device));
    DevState st;
    int s = read_state(c, &st);
    if (s) return s;
    if (global_speed) *global_speed = st.global_speed;
    if (speed_efficiency) *speed_efficiency = st.speed_efficiency;
    if (f_prev && c->n) {
        launch_gather_xy((int)c->n, c->b.ref_of, c->b.fprev, c->stage_xy, c->sA);
        CK(cudaMemcpyAsync(f_prev, c->stage_xy, (size_t)c->n * 8, cudaMemcpyDeviceToHost, c->sA));
        CK(cudaStreamSynchronize(c->sA));
    }
    return FA2_OK;
}

int fa2_set_force_params(fa2_ctx *c, float scale, float gravity) {
    if (!c) return FA2_ERR_INVALID_ARGUMENT;
    CK(cudaSetDevice(c->device));
    if (c->kp.k_r == scale && c->kp.k_g == gravity) return FA2_OK;
    CK(cudaStreamSynchronize(c->sA));
    c->kp.k_r = scale;
    c->kp.k_g = gravity;
    c->prm.scale = scale;
    c->prm.gravity = gravity;
    // the captured graphs hold the old values as kernel arguments
    drop_graphs(c);
    return FA2_OK;
}

int fa2_set_linlog(fa2_ctx *c, int32_t enable) {
    if (!c) return FA2_ERR_INVALID_ARGUMENT;
    CK(cudaSetDevice(c->device));
    if (c->kp.linlog == (enable != 0)) return FA2_OK;
    if (enable && c->kp.overlap) return FA2_ERR_UNSUPPORTED;
    CK(cudaStreamSynchronize(c->sA));
    c->kp.linlog = enable != 0;
    c->prm.linlog = enable != 0;
    drop_graphs(c);
    return FA2_OK;
}

int fa2_set_approximation(fa2_ctx *c, float theta, int32_t multipole) {
    if (!c || !(theta > 0.0f) || multipole < 1 || multipole > 2) return FA2_ERR_INVALID_ARGUMENT;
    CK(cudaSetDevice(c->device));
    const float itolsq = 1.0f / (theta * theta);  // src/RPForceAtlas2.cpp:47
    if (multipole >= 2 && c->kp.overlap) return FA2_ERR_UNSUPPORTED;
    if (c->kp.itolsq == itolsq && c->kp.multipole == multipole) {
        c->prm.theta = theta;
        return FA2_OK;
    }
    CK(cudaStreamSynchronize(c->sA));
    if (multipole >= 2) {
        const int s = ensure_quad_buffers(c);
        if (s) return s;
    }
    c->kp.itolsq = itolsq;
    c->kp.multipole = multipole;
    c->prm.theta = theta;
    c->prm.multipole = multipole;
    drop_graphs(c);  // theta and the walk variant are captured in the graphs
    return FA2_OK;
}

int fa2_exact_repulsion(fa2_ctx *c, int32_t n_samples, const uint32_t *samples, double *out) {
    if (!c || n_samples < 0 || (n_samples && (!samples || !out))) return FA2_ERR_INVALID_ARGUMENT;
    if (n_samples == 0) return FA2_OK;
    std::vector<uint32_t> internal(c->n);
    for (uint32_t k = 0; k < c->n; ++k) internal[c->ref_of[k]] = k;
    std::vector<uint32_t> ids((size_t)n_samples);
    for (int32_t s = 0; s < n_samples; ++s) {
        if (samples[s] >= c->n) return FA2_ERR_INVALID_ARGUMENT;
        ids[s] = internal[samples[s]];
    }
    CK(cudaSetDevice(c->device));
    uint32_t *d_ids = nullptr;
    double2 *d_out = nullptr;
    cudaError_t e = cudaMalloc(&d_ids, ids.size() * 4);
    if (e == cudaSuccess) e = cudaMalloc(&d_out, ids.size() * sizeof(double2));
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_ids, ids.data(), ids.size() * 4, cudaMemcpyHostToDevice, c->sA);
    if (e == cudaSuccess) {
        launch_exact_f64(c->b, c->kp, d_ids, n_samples, d_out, c->sA);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(out, d_out, ids.size() * sizeof(double2), cudaMemcpyDeviceToHost,
                            c->sA);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->sA);
    const int s = cuda_status(e);
    cudaFree(d_ids);
    cudaFree(d_out);
    return s;
}

const char *fa2_last_cuda_error(void) { return g_last_cuda_error; }

int fa2_set_accuracy_guard(fa2_ctx *c, int32_t every, int32_t n_samples) {
    if (!c || every < 0 || (every > 0 && n_samples <= 0)) return FA2_ERR_INVALID_ARGUMENT;
    // the guard's reference walk has no node sizes
    if (every > 0 && c->kp.overlap) return FA2_ERR_UNSUPPORTED;
    CK(cudaSetDevice(c->device));
    c->guard_checks = c->guard_fallbacks = 0;
    c->guard_err_cur = c->guard_err_plain = 0.0;
    if (every == 0 || c->n == 0) {
        c->guard_every = 0;
        return FA2_OK;
    }
    const int ns = (int)std::min<uint32_t>((uint32_t)n_samples, c->n);
    if (ns > c->guard_cap) {
        int s = FA2_OK;
        if ((s = dalloc(c, &c->guard_exact, (size_t)ns)) ||
            (s = dalloc(c, &c->guard_part, guard_part_count(ns))) ||
            (s = dalloc(c, &c->guard_plain, (size_t)ns)) ||
            (s = dalloc(c, &c->guard_cur, (size_t)ns)))
            return s;
        c->guard_cap = ns;
    }
    c->guard_every = every;
    c->guard_samples = ns;
    c->guard_left = every;
    return FA2_OK;
}

int fa2_get_accuracy_guard(fa2_ctx *c, double *err_current, double *err_plain, int32_t *checks,
                           int32_t *fallbacks) {
    if (!c) return FA2_ERR_INVALID_ARGUMENT;
    if (err_current) *err_current = c->guard_err_cur;
    if (err_plain) *err_plain = c->guard_err_plain;
    if (checks) *checks = c->guard_checks;
    if (fallbacks) *fallbacks = c->guard_fallbacks;
    return FA2_OK;
}

int fa2_set_prevent_overlap(fa2_ctx *c, const float *sizes) {
    if (!c) return FA2_ERR_INVALID_ARGUMENT;
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->sA));
    if (!sizes) {
        if (c->kp.overlap) {
            c->kp.overlap = 0;
            drop_graphs(c);
        }
        return FA2_OK;
    }
    if (c->kp.linlog || c->kp.multipole >= 2 || c->learn_on || c->guard_every > 0)
        return FA2_ERR_UNSUPPORTED;
    std::vector<float> internal(c->n);
    for (uint32_t i = 0; i < c->n; ++i) {
        const float v = sizes[c->ref_of[i]];
        if (!(v >= 0.0f) || !std::isfinite(v)) return FA2_ERR_INVALID_ARGUMENT;
        internal[i] = v;
    }
    if (c->n == 0) return FA2_OK;
    int s = FA2_OK;
    float *d_size = const_cast<float *>(c->b.size);
    if (!d_size && (s = dalloc(c, &d_size, c->n))) return s;
    if (!c->b.ssize && (s = dalloc(c, &c->b.ssize, c->n))) return s;
    c->b.size = d_size;
    CK(cudaMemcpyAsync(d_size, internal.data(), (size_t)c->n * 4, cudaMemcpyHostToDevice, c->sA));
    CK(cudaStreamSynchronize(c->sA));
    if (!c->kp.overlap) {
        c->kp.overlap = 1;
        drop_graphs(c);
    }
    return FA2_OK;
}

int fa2_set_overlap(fa2_ctx *c, int32_t enable) {
    if (!c) return FA2_ERR_INVALID_ARGUMENT;
    CK(cudaSetDevice(c->device));
    if (c->overlap == (enable != 0)) return FA2_OK;
    CK(cudaStreamSynchronize(c->sA));
    c->overlap = enable != 0;
    drop_graphs(c);  // recaptured with the new stream layout at the next step
    return FA2_OK;
}

// ------------------------------------------------ learned correction --

void fa2_mlp_init(fa2_mlp *mlp, uint32_t seed) {
    if (!mlp) return;
    mlp_default_init(mlp, seed);
}

int fa2_set_learned_correction(fa2_ctx *c, const fa2_mlp *mlp) {
    if (!c) return FA2_ERR_INVALID_ARGUMENT;
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->sA));
    if (!mlp) {
        if (c->learn_on) {
            c->learn_on = false;
            drop_graphs(c);
        }
        return FA2_OK;
    }
    if (!mlp_is_finite(*mlp)) return FA2_ERR_INVALID_ARGUMENT;
    if (c->kp.overlap) return FA2_ERR_UNSUPPORTED;
    mlp_blocks_per_sm();  // the launch shape, settled outside any graph capture
    int s = ensure_learn_buffers(c);
    if (s) return s;
    MlpDevice host;
    mlp_to_device(*mlp, host);
    CK(cudaMemcpyAsync(c->d_mlp, &host, sizeof(host), cudaMemcpyHostToDevice, c->sA));
    CK(cudaStreamSynchronize(c->sA));
    if (!c->learn_on) {
        c->learn_on = true;
        drop_graphs(c);  // the learned walk, MLP and tail are captured anew
    }
    return FA2_OK;
}

int fa2_mlp_launch_shape(int32_t device, int32_t *blocks_per_sm, int32_t *smem_bytes) {
    int nsm = 0;
    int s = use_device(device, &nsm);
    if (s) return s;
    const int nb = mlp_blocks_per_sm();
    if (blocks_per_sm) *blocks_per_sm = nb;
    if (smem_bytes) *smem_bytes = mlp_smem_bytes_host();
    return FA2_OK;
}

int fa2_mlp_forward(int32_t device, const fa2_mlp *mlp, const float *features, int64_t n,
                    float *out) {
    if (!mlp || n < 0 || (n && (!features || !out))) return FA2_ERR_INVALID_ARGUMENT;
    if (n == 0) return FA2_OK;
    int nsm = 0;
    int s = use_device(device, &nsm);
    if (s) return s;
    MlpDevice host;
    mlp_to_device(*mlp, host);
    DeviceScratch mem;
    MlpDevice *d_mlp = nullptr;
    float *d_feat = nullptr;
    float2 *d_out = nullptr;
    int *d_err = nullptr;
    if ((s = mem.get(&d_mlp, 1)) || (s = mem.get(&d_feat, (size_t)n * FA2_MLP_IN)) ||
        (s = mem.get(&d_out, (size_t)n)) || (s = mem.get(&d_err, 1)))
        return s;
    cudaStream_t st = mem.stream;
    CK(cudaMemcpyAsync(d_mlp, &host, sizeof(host), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(d_feat, features, (size_t)n * FA2_MLP_IN * 4, cudaMemcpyHostToDevice, st));
    CK(cudaMemsetAsync(d_err, 0, sizeof(int), st));
    launch_mlp_rows(d_mlp, d_feat, n, d_out, d_err, nsm, st);
    CK(cudaGetLastError());
    int err = 0;
    CK(cudaMemcpyAsync(out, d_out, (size_t)n * 8, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(&err, d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return err ? FA2_ERR_DEVICE_LIMIT : FA2_OK;
}

int fa2_mlp_train_step(int32_t device, fa2_mlp *params, fa2_mlp *adam_m, fa2_mlp *adam_v,
                       int32_t step, float lr, const float *features, const float *targets,
                       const float *weights, int32_t n, float *loss) {
    if (!params || !adam_m || !adam_v || step < 1 || n < 1 || !features || !targets || !weights)
        return FA2_ERR_INVALID_ARGUMENT;
    static_assert(sizeof(fa2_mlp) == sizeof(float) * kLearnParams, "fa2_mlp is the parameter vector");
    int nsm = 0;
    int s = use_device(device, &nsm);
    if (s) return s;
    DeviceScratch mem;
    float *d_p = nullptr, *d_m = nullptr, *d_v = nullptr, *d_x = nullptr, *d_w = nullptr,
          *d_scr = nullptr, *d_loss = nullptr;
    float2 *d_t = nullptr;
    if ((s = mem.get(&d_p, kLearnParams)) || (s = mem.get(&d_m, kLearnParams)) ||
        (s = mem.get(&d_v, kLearnParams)) || (s = mem.get(&d_x, (size_t)n * FA2_MLP_IN)) ||
        (s = mem.get(&d_t, (size_t)n)) || (s = mem.get(&d_w, (size_t)n)) ||
        (s = mem.get(&d_scr, learn_train_scratch_floats(n))) || (s = mem.get(&d_loss, 1)))
        return s;
    cudaStream_t st = mem.stream;
    CK(cudaMemcpyAsync(d_p, params, sizeof(fa2_mlp), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(d_m, adam_m, sizeof(fa2_mlp), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(d_v, adam_v, sizeof(fa2_mlp), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(d_x, features, (size_t)n * FA2_MLP_IN * 4, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(d_t, targets, (size_t)n * 8, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(d_w, weights, (size_t)n * 4, cudaMemcpyHostToDevice, st));
    launch_learn_train_step(d_p, d_m, d_v, step, lr, d_x, d_t, d_w, 1.0f, nullptr, n, d_scr,
                            d_loss, st);
    CK(cudaGetLastError());
    float l = 0.0f;
    CK(cudaMemcpyAsync(params, d_p, sizeof(fa2_mlp), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(adam_m, d_m, sizeof(fa2_mlp), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(adam_v, d_v, sizeof(fa2_mlp), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(&l, d_loss, sizeof(float), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (loss) *loss = l;
    return FA2_OK;
}

fa2_learn_set *fa2_learn_set_create(int32_t device, int64_t capacity, int *status) {
    int dummy;
    if (!status) status = &dummy;
    *status = FA2_ERR_INVALID_ARGUMENT;
    if (capacity < 1) return nullptr;
    int nsm = 0;
    if ((*status = use_device(device, &nsm))) return nullptr;
    fa2_learn_set *set = new fa2_learn_set();
    set->device = device;
    set->cap = capacity;
    const size_t cap = (size_t)capacity;
    if (cudaMalloc(&set->feat, cap * FA2_MLP_IN * 4) != cudaSuccess ||
        cudaMalloc(&set->tgt, cap * 8) != cudaSuccess ||
        cudaMalloc(&set->w, cap * 4) != cudaSuccess ||
        cudaStreamCreateWithFlags(&set->stream, cudaStreamNonBlocking) != cudaSuccess) {
        fa2_learn_set_destroy(set);
        *status = FA2_ERR_OUT_OF_MEMORY;
        return nullptr;
    }
    *status = FA2_OK;
    return set;
}

void fa2_learn_set_destroy(fa2_learn_set *set) {
    if (!set) return;
    cudaSetDevice(set->device);
    if (set->stream) cudaStreamSynchronize(set->stream);
    cudaFree(set->feat);
    cudaFree(set->tgt);
    cudaFree(set->w);
    cudaFree(set->st_feat);
    cudaFree(set->st_tgt);
    cudaFree(set->st_w);
    cudaFree(set->st_key);
    cudaFree(set->st_count);
    if (set->stream) cudaStreamDestroy(set->stream);
    delete set;
}

int64_t fa2_learn_set_size(const fa2_learn_set *set) { return set ? set->size : 0; }

int fa2_learn_collect(fa2_learn_set *set, fa2_ctx *c, float theta, int32_t multipole,
                      int64_t *added) {
    if (added) *added = 0;
    if (!set || !c || !(theta > 0.0f) || multipole < 1 || multipole > 2 ||
        set->device != c->device)
        return FA2_ERR_INVALID_ARGUMENT;
    CK(cudaSetDevice(c->device));
    if (c->n == 0) return FA2_OK;
    CK(cudaStreamSynchronize(c->sA));
    int s = multipole >= 2 ? ensure_quad_buffers(c) : FA2_OK;
    if (!s) s = ensure_learn_buffers(c);
    if (!s) s = set_staging(set, (int64_t)c->lb.seg_cap * kPairSegments);
    if (s) return s;
    Params kp = c->kp;
    kp.itolsq = 1.0f / (theta * theta);
    kp.multipole = multipole;
    Buffers b = c->b;
    b.sort_first = 0;  // every digit: the walk needs no earlier tree
    cudaStream_t A = c->sA;
    CK(cudaMemsetAsync(c->scratch, 0, c->scratch_bytes, A));
    CK(cudaMemsetAsync(set->st_count, 0, sizeof(unsigned long long), A));
    launch_keys(b, c->nsm, A);
    launch_sort(b, A);
    launch_tree_count(b, multipole >= 2, A);
    if (multipole >= 2) launch_moments(b, A);
    launch_emit(b, c->nsm, A);
    if (multipole >= 2) launch_quad_cells(b, c->nsm, A);
    launch_cell_a2(b, c->lb, c->nsm, A);
    launch_traverse_learn(b, kp, c->lb, c->trav_blocks, A);
    launch_learn_targets(b, kp, c->lb, set->st_feat, set->st_tgt, set->st_w, set->st_key,
                         set->st_count, (uint64_t)set->st_cap, c->nsm, A);
    CK(cudaGetLastError());
    DevState st;
    s = read_state(c, &st);
    if (s) return s;
    if (st.err) return FA2_ERR_DEVICE_LIMIT;
    if (st.poison) {
        // coincident bodies: the next step moves them apart; the flag goes
        // with this walk
        CK(cudaMemsetAsync(&c->b.st->poison, 0, sizeof(int), A));
        CK(cudaStreamSynchronize(A));
        return FA2_OK;
    }
    unsigned long long got = 0;
    CK(cudaMemcpy(&got, set->st_count, sizeof(got), cudaMemcpyDeviceToHost));
    const size_t k = (size_t)std::min<unsigned long long>(got, (unsigned long long)set->st_cap);
    if (k == 0) return FA2_OK;
    // the samples in (group, node) order, whatever order the warps wrote them in
    std::vector<uint64_t> key(k);
    std::vector<float> feat(k * FA2_MLP_IN), w(k);
    std::vector<float2> tgt(k);
    CK(cudaMemcpy(key.data(), set->st_key, k * 8, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(feat.data(), set->st_feat, k * FA2_MLP_IN * 4, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(tgt.data(), set->st_tgt, k * 8, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(w.data(), set->st_w, k * 4, cudaMemcpyDeviceToHost));
    std::vector<uint32_t> order(k);
    std::iota(order.begin(), order.end(), 0u);
    std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b2) { return key[a] < key[b2]; });
    const size_t room = (size_t)std::max<int64_t>(set->cap - set->size, 0);
    const size_t take = std::min(k, room);
    std::vector<float> feat2(take * FA2_MLP_IN), w2(take);
    std::vector<float2> tgt2(take);
    for (size_t q = 0; q < take; ++q) {
        const uint32_t o = order[q];
        std::copy(&feat[(size_t)o * FA2_MLP_IN], &feat[(size_t)o * FA2_MLP_IN] + FA2_MLP_IN,
                  &feat2[q * FA2_MLP_IN]);
        tgt2[q] = tgt[o];
        w2[q] = w[o];
    }
    if (take) {
        const size_t at = (size_t)set->size;
        CK(cudaMemcpy(set->feat + at * FA2_MLP_IN, feat2.data(), take * FA2_MLP_IN * 4,
                      cudaMemcpyHostToDevice));
        CK(cudaMemcpy(set->tgt + at, tgt2.data(), take * 8, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(set->w + at, w2.data(), take * 4, cudaMemcpyHostToDevice));
        set->size += (int64_t)take;
    }
    if (added) *added = (int64_t)take;
    return FA2_OK;
}

int fa2_learn_set_read(const fa2_learn_set *set, int64_t first, int64_t count, float *features,
                       float *targets, float *weights) {
    if (!set || first < 0 || count < 0 || first + count > set->size) return FA2_ERR_INVALID_ARGUMENT;
    if (count == 0) return FA2_OK;
    CK(cudaSetDevice(set->device));
    const size_t f0 = (size_t)first, k = (size_t)count;
    if (features)
        CK(cudaMemcpy(features, set->feat + f0 * FA2_MLP_IN, k * FA2_MLP_IN * 4,
                      cudaMemcpyDeviceToHost));
    if (targets) CK(cudaMemcpy(targets, set->tgt + f0, k * 8, cudaMemcpyDeviceToHost));
    if (weights) CK(cudaMemcpy(weights, set->w + f0, k * 4, cudaMemcpyDeviceToHost));
    return FA2_OK;
}

int fa2_learn_fit(fa2_learn_set *set, fa2_mlp *mlp, int32_t steps, int32_t batch, float lr,
                  uint32_t seed, float *final_loss) {
    if (!set || !mlp || steps < 1 || batch < 1 || !(lr > 0.0f) || set->size < 1)
        return FA2_ERR_INVALID_ARGUMENT;
    if (set->size > (int64_t)0xFFFFFFFFll) return FA2_ERR_TOO_LARGE;
    CK(cudaSetDevice(set->device));
    const int64_t size = set->size;
    const int bsz = (int)std::min<int64_t>(batch, size);
    cudaStream_t st = set->stream;
    DeviceScratch mem;
    float *d_p = nullptr, *d_m = nullptr, *d_v = nullptr, *d_scr = nullptr, *d_loss = nullptr;
    double *d_wsum = nullptr;
    uint32_t *d_idx = nullptr;
    int s = FA2_OK;
    if ((s = mem.get(&d_p, kLearnParams)) || (s = mem.get(&d_m, kLearnParams)) ||
        (s = mem.get(&d_v, kLearnParams)) || (s = mem.get(&d_scr, learn_train_scratch_floats(bsz))) ||
        (s = mem.get(&d_loss, 1)) || (s = mem.get(&d_wsum, 1)) ||
        (s = mem.get(&d_idx, (size_t)size)))
        return s;
    CK(cudaMemcpyAsync(d_p, mlp, sizeof(fa2_mlp), cudaMemcpyHostToDevice, st));
    CK(cudaMemsetAsync(d_m, 0, sizeof(fa2_mlp), st));
    CK(cudaMemsetAsync(d_v, 0, sizeof(fa2_mlp), st));
    launch_learn_weight_sum(set->w, (uint64_t)size, d_wsum, st);
    CK(cudaGetLastError());
    double wsum = 0.0;
    CK(cudaMemcpyAsync(&wsum, d_wsum, sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    const float wscale = wsum > 0.0 ? (float)((double)size / wsum) : 1.0f;
    std::vector<uint32_t> perm((size_t)size);
    std::iota(perm.begin(), perm.end(), 0u);
    std::mt19937 rng(seed);
    int64_t pos = size;  // forces a shuffle before the first batch
    for (int32_t t = 0; t < steps; ++t) {
        if (pos + bsz > size) {
            std::shuffle(perm.begin(), perm.end(), rng);
            CK(cudaStreamSynchronize(st));  // the last batch no longer reads d_idx
            CK(cudaMemcpyAsync(d_idx, perm.data(), (size_t)size * 4, cudaMemcpyHostToDevice, st));
            pos = 0;
        }
        const float lr_t =
            steps > 1 ? lr * (float)std::pow(0.05, (double)t / (double)(steps - 1)) : lr;
        launch_learn_train_step(d_p, d_m, d_v, t + 1, lr_t, set->feat, set->tgt, set->w, wscale,
                                d_idx + pos, bsz, d_scr, t + 1 == steps ? d_loss : nullptr, st);
        pos += bsz;
    }
    CK(cudaGetLastError());
    float l = 0.0f;
    CK(cudaMemcpyAsync(mlp, d_p, sizeof(fa2_mlp), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(&l, d_loss, sizeof(float), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (final_loss) *final_loss = l;
    return FA2_OK;
}

const char *fa2_status_string(int s) {
    switch (s) {
        case FA2_OK: return "ok";
        case FA2_ERR_INVALID_ARGUMENT: return "invalid argument";
        case FA2_ERR_NO_DEVICE: return "no usable CUDA device (sm_100 required)";
        case FA2_ERR_CUDA: return "CUDA runtime error";
        case FA2_ERR_OUT_OF_MEMORY: return "out of device memory";
        case FA2_ERR_DEVICE_LIMIT: return "device-side limit reached";
        case FA2_ERR_TOO_LARGE: return "graph too large for this engine";
        case FA2_ERR_UNSUPPORTED: return "unsupported option";
        case FA2_ERR_IO: return "file could not be read or written";
        default: return "unknown status";
    }
}

const char *fa2_version(void) { return "fa2b200 0.1 (sm_100a)"; }

}  // extern "C"
