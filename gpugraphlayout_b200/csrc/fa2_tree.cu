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
//   k_mom_*       (quadrupole option only) exact prefix sums of the bodies'
//   k_quad_cells  first and second moments, from which every cell's second
//                 moment follows the same way.
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

// An offset on the 2^-48 grid of k_tree_count moved to the 2^-44 grid of
// the moment sums (positions lie inside the root box, so |q| <= 2^44; the
// clamp only bounds the sums for inputs that do not).
__device__ __forceinline__ long long mom_grid(long long q48) {
    const long long q = q48 >> 4;
    constexpr long long kMax = 1ll << 45;
    return q > kMax ? kMax : (q < -kMax ? -kMax : q);
}

__global__ void __launch_bounds__(kCountThreads) k_tree_count(
    int n, const uint64_t *__restrict keys, int8_t *__restrict lcp, uint32_t *__restrict group,
    uint32_t *__restrict owner, uint32_t capacity, DevState *st, IterCounters *ctr,
    uint32_t *status,
    LookbackSums *__restrict lb, uint32_t *__restrict vals, float2 *__restrict pos,
    const float *__restrict mass, const uint32_t *__restrict ref_of,
    long long *__restrict pm, i128 *__restrict pxy, longlong2 *__restrict mom_q,
    uint32_t *__restrict mom_m) {
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
            // the quadrupole option's moment scan reads the bodies in this
            // order from here (2^-44 grid: the offset above >> 4)
            if (mom_q) {
                mom_q[k] = make_longlong2(mom_grid(qx[e]), mom_grid(qy[e]));
                mom_m[k] = (uint32_t)im[e];
            }
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
                    // give up on a wait that does not end, or at once when
                    // another tile has already given up
                    if (++spins > (1L << 22) ||
                        ((spins & 4095) == 0 && *((volatile int *)&st->err))) {
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

inline int grid_for(int n, int threads, int cap) {
    int g = (n + threads - 1) / threads;
    return g < 1 ? 1 : (g > cap ? cap : g);
}

// ------------------------------------------------------------ quadrupoles --

// The quadrupole option needs every cell's complex second moment about its
// centre of mass, a2 = sum m (z - Z)^2, the coefficient of the second term of
// its far field: sum_j m_j / (w - d_j) = M / w + a2 / w^3 + ..., w = z - Z,
// d_j = z_j - Z (the dipole term vanishes about Z).  As for the centres of
// mass, a cell's sums are two prefix differences over its run of sorted
// bodies: exact 128-bit prefix sums of m q, m q^2 on a 2^-44 root-radius grid
// (Moments), from a single-pass scan (k_mom_scan); k_quad_cells forms a2 per
// cell.

__device__ __forceinline__ void mom_add(Moments &a, const Moments &b) {
    a.x += b.x;
    a.y += b.y;
    a.re += b.re;
    a.im += b.im;
}

// a - b
__device__ __forceinline__ Moments mom_sub(const Moments &a, const Moments &b) {
    return Moments{a.x - b.x, a.y - b.y, a.re - b.re, a.im - b.im};
}

__device__ __forceinline__ Moments mom_shfl_up(const Moments &v, int o) {
    return Moments{shfl_up_i128(v.x, o), shfl_up_i128(v.y, o), shfl_up_i128(v.re, o),
                   shfl_up_i128(v.im, o)};
}

__device__ __forceinline__ Moments mom_shfl_xor(const Moments &v, int o) {
    return Moments{shfl_xor_i128(v.x, o), shfl_xor_i128(v.y, o), shfl_xor_i128(v.re, o),
                   shfl_xor_i128(v.im, o)};
}

constexpr double kMomScale = 17592186044416.0;  // 2^44

// Moments of one body from its grid offset and mass.
__device__ __forceinline__ Moments body_moments(longlong2 q, uint32_t m) {
    const i128 mx = (i128)(long long)m * q.x, my = (i128)(long long)m * q.y;
    return Moments{mx, my, mx * q.x - my * q.y, mx * q.y};
}

// The exclusive prefix of every sorted body's moments (pmom[k], and the total
// at pmom[n]) in one pass: tiles of kMomTile bodies taken in ticket order,
// each scanned in the block and offset by the tiles before it through a
// decoupled look-back (the scheme of k_tree_count).  A wait that does not end
// sets kErrScanWait.
__global__ void __launch_bounds__(kMomThreads) k_mom_scan(
    int n, const longlong2 *__restrict mq, const uint32_t *__restrict mm,
    MomLookback *__restrict lb, uint32_t *status, Moments *__restrict pmom, DevState *st,
    IterCounters *ctr) {
    __shared__ Moments s_w[kMomThreads / kWarp];
    __shared__ Moments s_prefix;
    __shared__ int s_tile;
    if (st->err || st->poison) return;
    if (threadIdx.x == 0) s_tile = (int)atomicAdd(&ctr->mom_ticket, 1u);
    __syncthreads();
    const int tile = s_tile;
    constexpr int kItems = kMomTile / kMomThreads;
    const int base = tile * kMomTile + threadIdx.x * kItems;
    longlong2 q[kItems];
    uint32_t m[kItems];
#pragma unroll
    for (int e = 0; e < kItems; ++e) {
        const bool in = base + e < n;
        q[e] = in ? mq[base + e] : make_longlong2(0, 0);
        m[e] = in ? mm[base + e] : 0u;
    }
    Moments run{0, 0, 0, 0};
#pragma unroll
    for (int e = 0; e < kItems; ++e) mom_add(run, body_moments(q[e], m[e]));
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    Moments inc = run;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const Moments t = mom_shfl_up(inc, o);
        if (lane >= o) mom_add(inc, t);
    }
    if (lane == 31) s_w[wid] = inc;
    __syncthreads();
    if (wid == 0) {
        Moments total{0, 0, 0, 0};
        if (lane == 0)
            for (int w = 0; w < kMomThreads / kWarp; ++w) {
                const Moments t = s_w[w];
                s_w[w] = total;
                mom_add(total, t);
            }
        const uint32_t kAgg = 1u, kPre = 2u;
        Moments prefix{0, 0, 0, 0};
        if (tile == 0) {
            if (lane == 0) {
                lb[0].incl = total;
                __threadfence();
                atomicExch(&status[0], kPre);
            }
        } else {
            if (lane == 0) {
                lb[tile].agg = total;
                __threadfence();
                atomicExch(&status[tile], kAgg);
            }
            // lane j reads the flag of tile hi - j: one round trip covers 32
            // earlier tiles, back to the nearest with an inclusive prefix
            int hi = tile - 1;
            long spins = 0;
            for (;;) {
                const int t = hi - lane;
                const uint32_t f = t >= 0 ? *((volatile uint32_t *)&status[t]) : kPre;
                const unsigned pre = __ballot_sync(kFull, f == kPre);
                const unsigned zero = __ballot_sync(kFull, f == 0);
                const int first = pre ? __ffs(pre) - 1 : 31;
                const unsigned need = first == 31 ? kFull : ((2u << first) - 1u);
                if (zero & need) {
                    // give up on a wait that does not end, or at once when
                    // another tile has already given up
                    if (++spins > (1L << 22) ||
                        ((spins & 4095) == 0 && *((volatile int *)&st->err))) {
                        if (lane == 0) atomicOr(&st->err, kErrScanWait);
                        break;
                    }
                    continue;
                }
                __threadfence();
                Moments v{0, 0, 0, 0};
                if (((need >> lane) & 1u) && t >= 0) {
                    const Moments *src = f == kPre ? &lb[t].incl : &lb[t].agg;
                    v.x = ldcg_i128(&src->x);
                    v.y = ldcg_i128(&src->y);
                    v.re = ldcg_i128(&src->re);
                    v.im = ldcg_i128(&src->im);
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) mom_add(v, mom_shfl_xor(v, o));
                mom_add(prefix, v);
                if (pre) break;
                hi -= 32;
            }
            if (lane == 0) {
                Moments incl = prefix;
                mom_add(incl, total);
                lb[tile].incl = incl;
                __threadfence();
                atomicExch(&status[tile], kPre);
            }
        }
        if (lane == 0) s_prefix = prefix;
    }
    __syncthreads();
    if (st->err) return;
    // this thread's exclusive prefix: earlier tiles, earlier warps, earlier lanes
    Moments pre = s_prefix;
    mom_add(pre, s_w[wid]);
    mom_add(pre, mom_sub(inc, run));
#pragma unroll
    for (int e = 0; e < kItems; ++e) {
        const int k = base + e;
        if (k >= n) break;
        pmom[k] = pre;
        mom_add(pre, body_moments(q[e], m[e]));
        if (k == n - 1) pmom[n] = pre;
    }
}

// a2 of the cell over sorted bodies k..b: exact integer sums about a grid
// point c near the centre of mass, then the centre's own offset in double.
__device__ __forceinline__ float2 cell_quadrupole(const Moments &hi, const Moments &lo,
                                                  long long mass, float radius) {
    const i128 M = mass;
    const Moments S = mom_sub(hi, lo);
    const double inv_m = 1.0 / (double)mass;
    const long long cx = __double2ll_rn(i128_to_double(S.x) * inv_m);
    const long long cy = __double2ll_rn(i128_to_double(S.y) * inv_m);
    // sum m ((q_x - c_x)^2 - (q_y - c_y)^2) and sum m (q_x - c_x)(q_y - c_y),
    // every term below 2^124
    const i128 tre = S.re - 2 * (i128)cx * S.x + 2 * (i128)cy * S.y +
                     ((i128)cx * cx - (i128)cy * cy) * M;
    const i128 tim = S.im - (i128)cx * S.y - (i128)cy * S.x + (i128)cx * cy * M;
    const double dx = i128_to_double(S.x - (i128)cx * M);
    const double dy = i128_to_double(S.y - (i128)cy * M);
    const double are = i128_to_double(tre) - (dx * dx - dy * dy) * inv_m;
    const double aim = i128_to_double(tim) - dx * dy * inv_m;
    const double u = (double)radius / kMomScale;
    return make_float2((float)(are * u * u), (float)(2.0 * aim * u * u));
}

// a2 of every cell.  A cell's bodies are the sorted run from its owner (the
// body that starts it) to the body at the last node of its subtree, the node
// before "next".  Each warp gathers the cells among 32 nodes at a time into a
// queue and works through it 32 cells at a time, so no lane idles on bodies.
constexpr int kQuadThreads = 256;

// 4 blocks per SM (64 registers); the launch puts no more than that on an SM
__global__ void __launch_bounds__(kQuadThreads, 4) k_quad_cells(const float4 *__restrict nodes,
                                                             const uint32_t *__restrict owner,
                                                             const long long *__restrict pm,
                                                             const Moments *__restrict pmom,
                                                             float2 *__restrict quad,
                                                             DevState *st) {
    __shared__ uint32_t s_q[kQuadThreads / kWarp][64];
    if (st->err || st->poison) return;
    const uint32_t total = st->tree_nodes;
    const float radius = st->radius;
    const int lane = threadIdx.x & 31;
    uint32_t *q = s_q[threadIdx.x >> 5];
    const uint32_t nwarps = gridDim.x * (kQuadThreads / kWarp);
    const uint32_t warp = blockIdx.x * (kQuadThreads / kWarp) + (threadIdx.x >> 5);
    auto one = [&](uint32_t g) {
        const uint32_t w = owner[g];
        const uint32_t next = meta_next(__float_as_int(nodes[g].w));
        const int k = (int)(w >> 6), b = (int)(owner[next - 1] >> 6);
        quad[g] = cell_quadrupole(pmom[b + 1], pmom[k], pm[b + 1] - pm[k], radius);
    };
    int cnt = 0;
    for (uint32_t c0 = warp * 32; c0 < total; c0 += nwarps * 32) {
        const uint32_t g = c0 + lane;
        const bool cell = g < total && (owner[g] & 63u) != 63u;
        const unsigned m = __ballot_sync(kFull, cell);
        if (cell) q[cnt + __popc(m & ((1u << lane) - 1u))] = g;
        cnt += __popc(m);
        __syncwarp();
        if (cnt >= 32) {
            one(q[lane]);
            const uint32_t rest = lane + 32 < cnt ? q[lane + 32] : 0;
            __syncwarp();
            if (lane + 32 < cnt) q[lane] = rest;
            cnt -= 32;
            __syncwarp();
        }
    }
    if (lane < cnt) one(q[lane]);
}

// ------------------------------------------------------------------- emit --

// One thread per tree node (grid-stride over the preorder index): a body
// writes its own record; a cell finds its last body, then forms its mass and
// centre of mass from the prefix sums at its two ends.  Node-parallel, so the
// body that starts many nested cells (body 0 starts one per level) spreads
// their searches over many threads.
// 8 blocks of 256 per SM (32 registers): the launch's up to 8 blocks per SM
// are all resident at once
__global__ void __launch_bounds__(256, 8) k_emit(int n, const uint64_t *__restrict keys,
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

}  // namespace

void launch_moments(const Buffers &b, cudaStream_t s) {
    k_mom_scan<<<mom_tiles(b.n), kMomThreads, 0, s>>>(b.n, b.mom_q, b.mom_m, b.mom_lb,
                                                      b.mom_status, b.pmom, b.st, b.ctr);
}

void launch_runs(const Buffers &b, int perturb, int nsm, cudaStream_t s) {
    k_runs<<<grid_for(b.n, 256, nsm * 8), 256, 0, s>>>(b.n, b.keys[0], b.vals[0], b.pos, b.ref_of,
                                                       b.st, perturb);
}

void launch_tree_count(const Buffers &b, bool keep_moments, cudaStream_t s) {
    k_tree_count<<<count_tiles(b.n), kCountThreads, 0, s>>>(
        b.n, b.keys[0], b.lcp, b.group, b.owner, b.capacity, b.st, b.ctr, b.count_status,
        b.lookback,
        b.vals[0], b.pos, b.mass, b.ref_of, b.pm, reinterpret_cast<i128 *>(b.pxy),
        keep_moments ? b.mom_q : nullptr, keep_moments ? b.mom_m : nullptr);
}

void launch_emit(const Buffers &b, int nsm, cudaStream_t s) {
    k_emit<<<grid_for(b.n, 256, nsm * 8), 256, 0, s>>>(
        b.n, b.keys[0], b.vals[0], b.lcp, b.group, b.owner, b.pos, b.mass, b.pm,
        reinterpret_cast<const i128 *>(b.pxy), b.nodes, b.body_node, b.st);
}

void launch_quad_cells(const Buffers &b, int nsm, cudaStream_t s) {
    k_quad_cells<<<grid_for(b.n, kQuadThreads, nsm * 4), kQuadThreads, 0, s>>>(
        b.nodes, b.owner, b.pm, b.pmom, b.quad, b.st);
}

}  // namespace fa2
