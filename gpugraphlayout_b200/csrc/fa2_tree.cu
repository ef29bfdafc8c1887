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

// Replays the cell centre of a 32-digit key path.
__device__ __forceinline__ void key_centre(uint64_t key, float rx, float ry, float rr, float &x,
                                           float &y, float &r) {
    x = rx;
    y = ry;
    r = rr;
    for (int lvl = 0; lvl < kLevels; ++lvl) {
        r *= 0.5f;
        const int j = (int)(key >> (2 * (kLevels - 1 - lvl))) & 3;
        x = __fadd_rn(x, (j & 1) ? r : -r);
        y = __fadd_rn(y, (j & 2) ? r : -r);
    }
}

// Orders two bodies that share all 32 digits by the digits below level 32
// (the reference keeps splitting: src/RPBHKernels.cu:282-313), then by
// reference id.  Returns true if a goes first.
__device__ bool deep_less(float2 pa, float2 pb, uint32_t ida, uint32_t idb, float x, float y,
                          float r) {
    for (int lvl = 0; lvl < kDeepLevels; ++lvl) {
        r *= 0.5f;
        const int ja = (x < pa.x ? 1 : 0) | (y < pa.y ? 2 : 0);
        const int jb = (x < pb.x ? 1 : 0) | (y < pb.y ? 2 : 0);
        if (ja != jb) return ja < jb;
        x = __fadd_rn(x, (ja & 1) ? r : -r);
        y = __fadd_rn(y, (ja & 2) ? r : -r);
    }
    return ida < idb;
}

// The run of equal keys that starts at sorted body k: order it, then either
// flag exactly coincident bodies (perturb == 0) or scale every body that sits
// on an earlier one (lower reference id) by .99, as the reference's insertion
// does for the later-inserted body (src/RPBHKernels.cu:271-278).
__device__ void fix_run(int k, int n, const uint64_t *__restrict keys, uint32_t *__restrict vals,
                        float2 *__restrict pos, const uint32_t *__restrict ref_of, DevState *st,
                        int perturb) {
    const uint64_t key = keys[k];
    int len = 2;
    while (k + len < n && keys[k + len] == key && len <= kMaxRun) ++len;
    if (len > kMaxRun) {
        atomicOr(&st->err, kErrRunTooLong);
        return;
    }
    float cx, cy, cr;
    key_centre(key, st->rootx, st->rooty, st->radius, cx, cy, cr);
    uint32_t *v = vals + k;
    for (int a = 1; a < len; ++a) {  // insertion sort, stable
        const uint32_t va = v[a];
        const float2 pa = pos[va];
        int b = a - 1;
        while (b >= 0) {
            const uint32_t vb = v[b];
            if (!deep_less(pa, pos[vb], ref_of[va], ref_of[vb], cx, cy, cr)) break;
            v[b + 1] = vb;
            --b;
        }
        v[b + 1] = va;
    }
    // coincident neighbours (equal positions are adjacent after ordering)
    bool any = false;
    float2 prev = pos[v[0]];
    for (int a = 1; a < len; ++a) {
        const float2 p = pos[v[a]];
        const bool same = p.x == prev.x && p.y == prev.y;
        prev = p;
        if (!same) continue;
        any = true;
        if (perturb) pos[v[a]] = make_float2((float)((double)p.x * .99), (float)((double)p.y * .99));
    }
    if (any && !perturb) atomicAdd(&st->poison, 1);
}

// Replay path: the runs of the last sort, with the .99 scaling applied.
__global__ void __launch_bounds__(256) k_runs(int n, const uint64_t *__restrict keys,
                                              uint32_t *__restrict vals, float2 *__restrict pos,
                                              const uint32_t *__restrict ref_of, DevState *st,
                                              int perturb) {
    if (st->err || st->poison) return;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k + 1 < n; k += gridDim.x * blockDim.x) {
        if (keys[k + 1] != keys[k] || (k > 0 && keys[k - 1] == keys[k])) continue;
        fix_run(k, n, keys, vals, pos, ref_of, st, perturb);
    }
}

// ------------------------------------------------------------- tree count --

__device__ __forceinline__ int lcp_at(const uint64_t *__restrict keys, int n, int k) {
    return (k < 0 || k >= n - 1) ? -1 : lcp_digits(keys[k], keys[k + 1]);
}

// cells that start at sorted body k
__device__ __forceinline__ int cells_at(int k, int Lk, int Lkm1) {
    return k == 0 ? max(Lk, 0) + 1 : max(0, Lk - Lkm1);
}

typedef __int128 i128;

__device__ __forceinline__ i128 shfl_up_i128(i128 v, int o) {
    const unsigned long long lo = (unsigned long long)v;
    const long long hi = (long long)(v >> 64);
    const unsigned long long lo2 = __shfl_up_sync(kFull, lo, o);
    const long long hi2 = __shfl_up_sync(kFull, hi, o);
    return ((i128)hi2 << 64) | (i128)lo2;
}

__device__ __forceinline__ i128 shfl_xor_i128(i128 v, int o) {
    const unsigned long long lo = (unsigned long long)v;
    const long long hi = (long long)(v >> 64);
    const unsigned long long lo2 = __shfl_xor_sync(kFull, lo, o);
    const long long hi2 = __shfl_xor_sync(kFull, hi, o);
    return ((i128)hi2 << 64) | (i128)lo2;
}

// 128-bit load that bypasses L1 (the value was written by another block)
__device__ __forceinline__ i128 ldcg_i128(const i128 *p) {
    const longlong2 v = __ldcg(reinterpret_cast<const longlong2 *>(p));
    return ((i128)v.y << 64) | (i128)(unsigned long long)v.x;
}

__device__ __forceinline__ double i128_to_double(i128 v) {
    const long long hi = (long long)(v >> 64);
    const unsigned long long lo = (unsigned long long)v;
    return (double)hi * 18446744073709551616.0 + (double)lo;
}

// Fixed-point offset from the root centre, in 2^-48 root radii (finer than a
// float32 ulp of any coordinate but the tiniest), kept within +-2^55 (a body
// scaled by .99 may sit outside the box); mass (< 2^24) x offset is formed in
// 128 bits and a sum over 2^25 bodies stays below 2^105.
constexpr double kFixedScale = 281474976710656.0;  // 2^48
__device__ __forceinline__ long long fixed_offset(float p, float root, double scale) {
    double q = ((double)p - (double)root) * scale;
    q = fmin(fmax(q, -36028797018963968.0), 36028797018963968.0);
    return __double2ll_rn(q);
}

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
        if (run_starts & (1u << e)) fix_run(base + e, n, keys, vals, pos, ref_of, st, 0);
}

// ------------------------------------------------------------------- emit --

__device__ __forceinline__ int load_lcp(const int8_t *__restrict lcp, int n, int k) {
    return (k < 0 || k >= n - 1) ? -1 : (int)lcp[k];
}

// preorder index of sorted body b
__device__ __forceinline__ uint32_t body_index(const int8_t *__restrict lcp,
                                               const uint32_t *__restrict group, int n, int b) {
    const int Lb = load_lcp(lcp, n, b), Lbm1 = load_lcp(lcp, n, b - 1);
    return group[b] + (uint32_t)cells_at(b, Lb, Lbm1);
}

// Last body of the cell at level lvl that starts at sorted body k: the first
// j >= k with L[j] < lvl.  Small cells end within a few bodies (a short scan
// of L); larger ones are found by exponential + binary search over the keys
// (LCP(K_k, K_j) falls as j grows).
__device__ int find_end(const uint64_t *__restrict keys, const int8_t *__restrict lcp, int n,
                        int k, int lvl) {
    constexpr int kScan = 8;
    int L[kScan];
#pragma unroll
    for (int s = 0; s < kScan; ++s) L[s] = load_lcp(lcp, n, k + s);
#pragma unroll
    for (int s = 0; s < kScan; ++s)
        if (L[s] < lvl) return k + s;
    const uint64_t kk = keys[k];
    int ok = k + kScan - 1, step = 1, bad = n;
    for (;;) {
        const int j = ok + step;
        if (j >= n) {
            bad = n;
            break;
        }
        if (lcp_digits(keys[j], kk) >= lvl) {
            ok = j;
            step <<= 1;
        } else {
            bad = j;
            break;
        }
    }
    int lo = ok, hi = bad - 1;  // largest j with LCP(K_k, K_j) >= lvl, in [ok, bad)
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (lcp_digits(keys[mid], kk) >= lvl)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

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
