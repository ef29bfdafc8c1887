// fa2_tree.cu -- quadtree build from the sorted Morton keys.
//
// The reference inserts bodies into its quadtree with locks
// (TreeBuildingKernel, src/RPBHKernels.cu:184-329) and sums cells bottom-up
// with spin-waits (SummarizationKernel, :357-506).  The tree's shape does not
// depend on insertion order: its cells are exactly the quadrant prefixes that
// hold at least two bodies.  With the bodies sorted by key (the reference's
// in-order sortd), body k starts the cells at levels L[k-1]+1 .. L[k], where
// L[k] is the number of leading digits keys k and k+1 share.  So:
//
//   k_tree_count  L[k], the number of nodes each body contributes (its cells
//                 plus itself), and one single-pass scan over the sorted
//                 bodies that gives every node its preorder index and, in the
//                 same pass, exact prefix sums of mass and mass x position
//                 (integers: mass is degree + 1; positions in 2^-48 steps of
//                 the root radius; 128-bit sums), so any cell's mass and centre
//                 of mass are two prefix differences.  Each node's owner (the
//                 body that starts it) is recorded.  It also orders runs of
//                 equal 64-bit keys (trees deeper than 32 levels) and flags
//                 exactly coincident bodies.
//   k_emit        writes every node once, one thread per node: bodies from
//                 their positions; cells
//                 with level, mass, centre of mass (prefix differences over
//                 the cell's body range) and the index of the node after their
//                 subtree.  No parent links, atomics or fences are needed.
//
// Against the reference's float summation in quadrant order
// (src/RPBHKernels.cu:461-494) the centres agree to float rounding; the sums
// here are exact and do not depend on thread timing.
#include <stdint.h>

#include "fa2_device.cuh"

namespace fa2 {

namespace {

constexpr unsigned kFull = kFullMask;

// ------------------------------------------------------------------- runs --

// Replay path: the runs of the last sort, with the .99 scaling applied.
__global__ void __launch_bounds__(256) k_runs(int n, const uint64_t *__restrict keys,
                                              uint32_t *__restrict vals, float2 *__restrict pos,
                                              const uint32_t *__restrict ref_of, DevState *st,
                                              int perturb) {
    if (st->err || st->poison) return;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k + 1 < n; k += gridDim.x * blockDim.x) {
        if (keys[k + 1] != keys[k] || (k > 0 && keys[k - 1] == keys[k])) continue;
        fix_run(k, n, keys, vals, pos, ref_of, st->rootx, st->rooty, st->radius, &st->err,
                &st->poison, perturb);
    }
}

// ------------------------------------------------------------- tree count --

struct NodeSums {
    uint32_t g;  // nodes (cells + body)
    long long m;
    i128 x, y;
};

__device__ __forceinline__ void sums_add(NodeSums &a, const NodeSums &b) {
    a.g += b.g;
    a.m += b.m;
    a.x += b.x;
    a.y += b.y;
}

__global__ void __launch_bounds__(kCountThreads) k_tree_count(
    int n, const uint64_t *__restrict keys, int8_t *__restrict lcp, uint32_t *__restrict group,
    uint32_t *__restrict owner, uint32_t capacity, DevState *st, IterCounters *ctr,
    uint32_t *status,
    LookbackSums *__restrict lb, uint32_t *__restrict vals, float2 *__restrict pos,
    const float *__restrict mass, const uint32_t *__restrict ref_of,
    long long *__restrict pm, i128 *__restrict pxy) {
    __shared__ int s_tile;
    __shared__ NodeSums s_warp[kCountThreads / kWarp];
    __shared__ NodeSums s_prefix;
    if (st->err || st->poison) return;
    if (threadIdx.x == 0) s_tile = atomicAdd(&ctr->count_ticket, 1u);
    __syncthreads();
    const int tile = s_tile;
    const int base = tile * kCountTile + threadIdx.x * kCountItems;
    const double scale = st->radius > 0.0f ? kFixedScale / (double)st->radius : 1.0;
    const float rx = st->rootx, ry = st->rooty;
    int g[kCountItems];
    long long im[kCountItems], qx[kCountItems], qy[kCountItems];
    uint32_t run_starts = 0;
    NodeSums sum{0, 0, 0, 0};
#pragma unroll
    for (int e = 0; e < kCountItems; ++e) {
        const int k = base + e;
        g[e] = 0;
        im[e] = qx[e] = qy[e] = 0;
        if (k < n) {
            const int Lk = lcp_at(keys, n, k);
            const int Lkm1 = lcp_at(keys, n, k - 1);
            lcp[k] = (int8_t)Lk;
            g[e] = cells_at(k, Lk, Lkm1) + 1;
            // a run of equal 64-bit keys starts here (trees past depth 32)
            if (Lk == kLevels && Lkm1 != kLevels) run_starts |= 1u << e;
            const uint32_t i = vals[k];
            const float2 p = pos[i];
            im[e] = (long long)mass[i];
            qx[e] = fixed_offset(p.x, rx, scale);
            qy[e] = fixed_offset(p.y, ry, scale);
        }
        sum.g += (uint32_t)g[e];
        sum.m += im[e];
        sum.x += (i128)im[e] * qx[e];
        sum.y += (i128)im[e] * qy[e];
    }
    // block exclusive scan of the per-thread sums
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    NodeSums inc = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        NodeSums t;
        t.g = __shfl_up_sync(kFull, inc.g, o);
        t.m = __shfl_up_sync(kFull, inc.m, o);
        t.x = shfl_up_i128(inc.x, o);
        t.y = shfl_up_i128(inc.y, o);
        if (lane >= o) sums_add(inc, t);
    }
    if (lane == 31) s_warp[wid] = inc;
    __syncthreads();
    if (wid == 0) {
        NodeSums run{0, 0, 0, 0};
        if (lane == 0) {
            for (int w = 0; w < kCountThreads / kWarp; ++w) {
                const NodeSums t = s_warp[w];
                s_warp[w] = run;
                sums_add(run, t);
            }
        }
        // Decoupled look-back over tiles: the flag word holds the node count,
        // the mass sums sit beside it and are written before the flag.  The
        // whole warp looks back: lane j reads the flag of tile (hi - j), so
        // one round trip covers 32 earlier tiles.  The tiles needed are those
        // from the nearest one with an inclusive prefix up to this one.
        const uint32_t kAgg = 1u << 30, kPre = 2u << 30, kMask = (1u << 30) - 1;
        NodeSums prefix{0, 0, 0, 0};
        if (tile == 0) {
            if (lane == 0) {
                lb[0].incl_m = run.m;
                lb[0].incl_x = run.x;
                lb[0].incl_y = run.y;
                __threadfence();
                atomicExch(&status[0], kPre | run.g);
            }
        } else {
            if (lane == 0) {
                lb[tile].agg_m = run.m;
                lb[tile].agg_x = run.x;
                lb[tile].agg_y = run.y;
                __threadfence();
                atomicExch(&status[tile], kAgg | run.g);
            }
            int hi = tile - 1;
            long spins = 0;
            for (;;) {
                const int t = hi - lane;
                // tile 0 always ends with an inclusive prefix, so a lane past
                // it is never needed
                const uint32_t s = t >= 0 ? *((volatile uint32_t *)&status[t]) : kPre;
                const unsigned pre = __ballot_sync(kFull, (s >> 30) == 2);
                const unsigned zero = __ballot_sync(kFull, (s >> 30) == 0);
                const int first = pre ? __ffs(pre) - 1 : 31;
                const unsigned need = first == 31 ? kFull : ((2u << first) - 1u);
                if (zero & need) {
                    if (++spins > (1L << 22)) {
                        if (lane == 0) atomicOr(&st->err, kErrScanWait);
                        break;
                    }
                    continue;
                }
                __threadfence();
                NodeSums v{0, 0, 0, 0};
                if (((need >> lane) & 1u) && t >= 0) {
                    v.g = s & kMask;
                    if ((s >> 30) == 2) {
                        v.m = __ldcg(&lb[t].incl_m);
                        v.x = ldcg_i128(&lb[t].incl_x);
                        v.y = ldcg_i128(&lb[t].incl_y);
                    } else {
                        v.m = __ldcg(&lb[t].agg_m);
                        v.x = ldcg_i128(&lb[t].agg_x);
                        v.y = ldcg_i128(&lb[t].agg_y);
                    }
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    v.g += __shfl_xor_sync(kFull, v.g, o);
                    v.m += __shfl_xor_sync(kFull, v.m, o);
                    v.x += shfl_xor_i128(v.x, o);
                    v.y += shfl_xor_i128(v.y, o);
                }
                sums_add(prefix, v);
                if (pre) break;
                hi -= 32;
            }
            if (lane == 0) {
                NodeSums incl = prefix;
                sums_add(incl, run);
                lb[tile].incl_m = incl.m;
                lb[tile].incl_x = incl.x;
                lb[tile].incl_y = incl.y;
                __threadfence();
                atomicExch(&status[tile], kPre | incl.g);
            }
        }
        if (lane == 0) s_prefix = prefix;
    }
    __syncthreads();
    NodeSums off = s_prefix;
    sums_add(off, s_warp[wid]);
    // exclusive offset of this thread = prefix + warp offset + lanes before
    off.g += inc.g - sum.g;
    off.m += inc.m - sum.m;
    off.x += inc.x - sum.x;
    off.y += inc.y - sum.y;
#pragma unroll
    for (int e = 0; e < kCountItems; ++e) {
        const int k = base + e;
        if (k < n) {
            group[k] = off.g;
            pm[k] = off.m;
            pxy[2 * (size_t)k] = off.x;
            pxy[2 * (size_t)k + 1] = off.y;
            // the owner of each node body k starts: its cells, then itself
            const uint32_t c = (uint32_t)g[e] - 1u;
            for (uint32_t q = 0; q <= c; ++q) {
                const uint32_t idx = off.g + q;
                if (idx < capacity) owner[idx] = ((uint32_t)k << 6) | (q < c ? q : 63u);
            }
        }
        off.g += (uint32_t)g[e];
        off.m += im[e];
        off.x += (i128)im[e] * qx[e];
        off.y += (i128)im[e] * qy[e];
        if (k == n - 1) {
            pm[n] = off.m;
            pxy[2 * (size_t)n] = off.x;
            pxy[2 * (size_t)n + 1] = off.y;
            st->tree_nodes = off.g;
            st->max_level = 0;     // raised by k_emit
            st->interactions = 0;  // counted by k_traverse
            st->visits = 0;
            if (off.g > capacity) atomicOr(&st->err, kErrTreeTooLarge);
        }
    }
    // after this tile's offsets are published, so a long run delays no one
#pragma unroll
    for (int e = 0; e < kCountItems; ++e)
        if (run_starts & (1u << e)) fix_run(base + e, n, keys, vals, pos, ref_of, st->rootx, st->rooty, st->radius,
                    &st->err, &st->poison, 0);
}

// ------------------------------------------------------------------- emit --

// One thread per tree node (grid-stride over the preorder index): a body
// writes its own record; a cell finds its last body, then forms its mass and
// centre of mass from the prefix sums at its two ends.  Node-parallel, so the
// body that starts many nested cells (body 0 starts one per level) spreads
// their searches over many threads.
__global__ void __launch_bounds__(256) k_emit(int n, const uint64_t *__restrict keys,
                                              const uint32_t *__restrict vals,
                                              const int8_t *__restrict lcp,
                                              const uint32_t *__restrict group,
                                              const uint32_t *__restrict owner,
                                              const float2 *__restrict pos,
                                              const float *__restrict mass,
                                              const long long *__restrict pm,
                                              const i128 *__restrict pxy,
                                              float4 *__restrict nodes,
                                              uint32_t *__restrict body_node, DevState *st) {
    if (st->err || st->poison) return;
    const uint32_t total = st->tree_nodes;
    const double inv_scale = st->radius > 0.0f ? (double)st->radius / kFixedScale : 1.0;
    const double rx = st->rootx, ry = st->rooty;
    int local_max = 0;
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < total;
         g += gridDim.x * blockDim.x) {
        const uint32_t w = owner[g];
        const int k = (int)(w >> 6), q = (int)(w & 63u);
        if (q == 63) {
            const uint32_t i = vals[k];
            const float2 p = pos[i];
            nodes[g] = make_float4(p.x, p.y, mass[i], make_meta(g + 1, kBodyLevel));
            body_node[k] = g;
            continue;
        }
        // the cells that start at body k have levels lo .. lo + c - 1
        const int lvl = (k == 0 ? 0 : load_lcp(lcp, n, k - 1) + 1) + q;
        const int b = lvl == 0 ? n - 1 : find_end(keys, lcp, n, k, lvl);
        const uint32_t next = body_index(lcp, group, n, b) + 1;
        const double cm = (double)(pm[b + 1] - pm[k]);
        const double sx = i128_to_double(pxy[2 * (size_t)(b + 1)] - pxy[2 * (size_t)k]);
        const double sy = i128_to_double(pxy[2 * (size_t)(b + 1) + 1] - pxy[2 * (size_t)k + 1]);
        nodes[g] = make_float4((float)(rx + sx / cm * inv_scale), (float)(ry + sy / cm * inv_scale),
                               (float)cm, make_meta(next, lvl));
        local_max = max(local_max, lvl);
    }
    local_max = __reduce_max_sync(kFull, local_max);
    if ((threadIdx.x & 31) == 0 && local_max > 0) atomicMax(&st->max_level, local_max);
}

inline int grid_for(int n, int threads, int cap) {
    int g = (n + threads - 1) / threads;
    return g < 1 ? 1 : (g > cap ? cap : g);
}

}  // namespace

void launch_runs(const Buffers &b, int perturb, int nsm, cudaStream_t s) {
    k_runs<<<grid_for(b.n, 256, nsm * 8), 256, 0, s>>>(b.n, b.keys[0], b.vals[0], b.pos, b.ref_of,
                                                       b.st, perturb);
}

void launch_tree_count(const Buffers &b, cudaStream_t s) {
    k_tree_count<<<count_tiles(b.n), kCountThreads, 0, s>>>(
        b.n, b.keys[0], b.lcp, b.group, b.owner, b.capacity, b.st, b.ctr, b.count_status,
        b.lookback,
        b.vals[0], b.pos, b.mass, b.ref_of, b.pm, reinterpret_cast<i128 *>(b.pxy));
}

void launch_emit(const Buffers &b, int nsm, cudaStream_t s) {
    k_emit<<<grid_for(b.n, 256, nsm * 8), 256, 0, s>>>(
        b.n, b.keys[0], b.vals[0], b.lcp, b.group, b.owner, b.pos, b.mass, b.pm,
        reinterpret_cast<const i128 *>(b.pxy), b.nodes, b.body_node, b.st);
}

}  // namespace fa2
