// fa2_kernels.cu -- the per-iteration kernels of the B200 ForceAtlas2 engine
// around the quadtree: bounding box, Morton keys, force traversal (+ speed),
// displacement, attraction, and the id permutations of the C ABI.  The radix
// sort is in fa2_sort.cu, the tree build in fa2_tree.cu.
//
// Keys: each body's 32 quadrant digits, computed with the reference's float
// cell-centre arithmetic and tie rule (src/RPBHKernels.cu:217-241), form a
// 64-bit Morton key; keys ascending give the reference's in-order body order
// (sortd).  The tree is stored in preorder with each node's "next" index (the
// node after its subtree), so the traversal needs no stack.
#include <float.h>
#include <stdint.h>

#include "fa2_device.cuh"
#include "fa2_learn.cuh"

namespace fa2 {

namespace {

constexpr unsigned kFull = 0xffffffffu;

// ------------------------------------------------------------------- bbox --

__device__ __forceinline__ float4 bbox_merge(float4 a, float4 b) {
    return make_float4(fminf(a.x, b.x), fmaxf(a.y, b.y), fminf(a.z, b.z), fmaxf(a.w, b.w));
}

__device__ __forceinline__ float4 warp_bbox(float4 a) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        float4 b;
        b.x = __shfl_xor_sync(kFull, a.x, o);
        b.y = __shfl_xor_sync(kFull, a.y, o);
        b.z = __shfl_xor_sync(kFull, a.z, o);
        b.w = __shfl_xor_sync(kFull, a.w, o);
        a = bbox_merge(a, b);
    }
    return a;
}

// Block bounding box (minx, maxx, miny, maxy) of the thread values; the
// last block to finish merges all block results and sets the root cell the
// way BoundingBoxKernel does (src/RPBHKernels.cu:128-148).  Every thread of
// the block must call it.  A thread that saw a NaN or infinite position
// passes bad: the next iteration then stops with kErrNonFinite instead of
// building a tree from it.
template <int THREADS>
__device__ void bbox_finish(float4 a, bool bad, float4 *__restrict partial, unsigned *done,
                            DevState *st) {
    __shared__ float4 s_w[THREADS / kWarp];
    __shared__ bool s_last;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (__any_sync(kFull, bad) && lane == 0) atomicOr(&st->err, kErrNonFinite);
    a = warp_bbox(a);
    if (lane == 0) s_w[wid] = a;
    __syncthreads();
    if (threadIdx.x == 0) {
        float4 b = s_w[0];
        for (int w = 1; w < THREADS / kWarp; ++w) b = bbox_merge(b, s_w[w]);
        partial[blockIdx.x] = b;
        __threadfence();
        s_last = atomicAdd(done, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    a = make_float4(FLT_MAX, -FLT_MAX, FLT_MAX, -FLT_MAX);
    for (int b = threadIdx.x; b < (int)gridDim.x; b += THREADS) a = bbox_merge(a, __ldcg(&partial[b]));
    a = warp_bbox(a);
    __syncthreads();
    if (lane == 0) s_w[wid] = a;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < THREADS / kWarp; ++w) a = bbox_merge(a, s_w[w]);
        st->minx = a.x;
        st->maxx = a.y;
        st->miny = a.z;
        st->maxy = a.w;
        st->radius = fmaxf(a.y - a.x, a.w - a.z) * 0.5f;
        st->rootx = (a.x + a.y) * 0.5f;
        st->rooty = (a.z + a.w) * 0.5f;
    }
}

// Bounding box of the current positions (run after positions are set from
// the host; during stepping the displacement pass computes it).
__global__ void __launch_bounds__(kBBoxThreads) k_bbox(int n, const float2 *__restrict pos,
                                                       float4 *__restrict partial,
                                                       DevState *st, IterCounters *ctr) {
    float4 a = make_float4(FLT_MAX, -FLT_MAX, FLT_MAX, -FLT_MAX);
    bool bad = false;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float2 p = pos[i];
        a = bbox_merge(a, make_float4(p.x, p.x, p.y, p.y));
        bad |= !(isfinite(p.x) && isfinite(p.y));
    }
    bbox_finish<kBBoxThreads>(a, bad, partial, &ctr->bbox_done, st);
}

// Whether a learned walk keeps an accepted cell as a pair: its size h is at
// least kLearnMinRatio theta of its distance (wx, wy) from the group's
// centroid.  With the cell's threshold dq = (2h)^2 / theta^2 + eps,
// h / d >= c theta  <=>  dq - eps >= 4 c^2 d^2: no theta needed.
__device__ __forceinline__ bool learn_keep(float dq, float wx, float wy, float eps) {
    return dq - eps >= 4.0f * kLearnMinRatio * kLearnMinRatio * (wx * wx + wy * wy);
}

// ------------------------------------------------------------------- keys --

// One block per sort tile: the tile's keys, the tile's counts of the digit
// of the first sort pass (that pass's per-tile input) and the tile's share of
// the digit histograms of all eight passes (order-independent, so counted
// once here).
__global__ void __launch_bounds__(1024) k_keys(int n, int tile, int first,
                                              const float2 *__restrict pos,
                                              const DevState *__restrict st,
                                              uint64_t *__restrict keys, uint32_t *__restrict vals,
                                              IterCounters *ctr, uint32_t *__restrict counts) {
    __shared__ unsigned s_hist[8][256];
    if (st->err || st->poison) return;
    for (int j = threadIdx.x; j < 8 * 256; j += blockDim.x) (&s_hist[0][0])[j] = 0;
    __syncthreads();
    const float rx = st->rootx, ry = st->rooty, rr = st->radius;
    const int tile0 = blockIdx.x * tile;
    const int tile_end = min(n, tile0 + tile);
    for (int i = tile0 + threadIdx.x; i < tile_end; i += blockDim.x) {
        float2 p = pos[i];
        uint64_t key = morton_key(p.x, p.y, rx, ry, rr);
        keys[i] = key;
        vals[i] = (uint32_t)i;
        // the histograms of the passes the sort runs
        for (int ps = first; ps < 8; ++ps) atomicAdd(&s_hist[ps][(key >> (8 * ps)) & 255], 1u);
    }
    __syncthreads();
    for (int j = threadIdx.x; j < 8 * 256; j += blockDim.x) {
        unsigned c = (&s_hist[0][0])[j];
        if ((j >> 8) == first)
            counts[((size_t)first * gridDim.x + blockIdx.x) * 256 + (j & 255)] = c;
        if (c) atomicAdd(&(&ctr->hist[0][0])[j], c);
    }
}

// --------------------------------------------------------------- traverse --

// Repulsion by a warp-cooperative preorder walk.  The 32 lanes of a warp
// hold 32 consecutive bodies of the sorted order, as the reference's
// ForceCalculationKernel does (src/RPBHKernels.cu:609-685); a cell is used as
// a whole only if every lane passes d^2 + eps >= dq[level] (:661), else the
// warp descends into it.  Bodies always interact.  The walk visits nodes in
// the reference's order, so each lane adds the same terms in the same order.
// The tail adds gravity + attraction, forms the swing and traction sums
// (SpeedKernel, src/RPFA2Kernels.cu:111-202) and, in the last block to
// finish, updates the adaptive speed (:204-219).
//
// QUAD adds, for every accepted cell, the quadrupole term of its far field,
// conj(a2 / w^3) = conj(a2) u^3 with w = z - Z, u = w / |w|^2 and the softened
// |w|^2 = d^2 + eps; a2 is the cell's complex second moment (k_quad_cells).  No
// reference counterpart: it is the option fa2_set_approximation selects.
//
// LEARN (the learned correction, fa2_learn.cuh) also records, per group, the
// centroid and second moments of its bodies and the cells the whole group
// accepted that are not small for their distance (a (group, node) pair,
// gathered 32 at a time in registers, one per lane, and tested with
// learn_keep when the 32 are written out), and
// writes each body's repulsion in sorted order instead of the tail: the MLP
// and k_learn_tail finish the iteration.  The sums are the same.
//
// OVERLAP (prevent_overlap, with the monopole walk) repels accepted bodies by
// the paper's anti-collision rule (overlap_factor) with the sizes of the
// sorted bodies in ssize; a body node's sorted index is its owner's.
template <bool QUAD, bool LEARN, bool OVERLAP = false>
__global__ void __launch_bounds__(kTravThreads, 2048 / kTravThreads) k_traverse(
    int n, const float4 *__restrict nodes, const float2 *__restrict quad,
    const uint32_t *__restrict body_node,
    const uint32_t *__restrict vals, const float2 *__restrict fag,
    const float2 *__restrict fprev, float2 *__restrict f, float2 *__restrict warp_partial,
    DevState *st, IterCounters *ctr, Params prm, LearnBuffers lb,
    const uint32_t *__restrict owner = nullptr, const float *__restrict ssize = nullptr) {
    __shared__ float s_dq[64];
    __shared__ bool s_last;
    __shared__ float s_red[2][kTravThreads / kWarp];
    if (st->err || st->poison) return;
    if (threadIdx.x == 0) {
        // src/RPBHKernels.cu:579-592: dq for the children of the root is
        // (2 radius)^2 / theta^2 + eps, quartering per level.
        float tmp = st->radius * 2;
        float dq = tmp * tmp * prm.itolsq;
        s_dq[0] = 0.0f;
        for (int l = 1; l <= kLevels; ++l) {
            s_dq[l] = dq + prm.epssq;
            dq = dq * 0.25f;
        }
        for (int l = kLevels + 1; l < 64; ++l) s_dq[l] = 0.0f;
        if (blockIdx.x == 0) st->trav_radius = st->radius;
    }
    __syncthreads();
    const uint32_t end = st->tree_nodes;
    const int lane = threadIdx.x & 31;
    const int nwarps = (n + 31) >> 5;
    // Groups of 32 bodies are handed out one at a time from a global ticket:
    // the work per group varies with the local density of the layout, and
    // warps that take consecutive tickets walk neighbouring bodies, so the
    // nodes they load are shared in L2.
    for (;;) {
        int w = 0;
        if (lane == 0) w = (int)atomicAdd(&ctr->trav_ticket, 1u);
        w = __shfl_sync(kFull, w, 0);
        if (w >= nwarps) break;
        const int k = w * 32 + lane;
        const bool active = k < n;
        const float4 me = nodes[body_node[active ? k : n - 1]];
        // a lane without a body sits far away: it passes every test and its
        // (unused) sums never feed anything
        const float px = active ? me.x : 1e30f, py = active ? me.y : 1e30f;
        const float my_size = OVERLAP && active ? ssize[k] : 0.0f;
        // sum of m_j d / (d^2 + eps) over the accepted nodes; the body's own
        // k_r m_i multiplies the sum once at the end
        float ax = 0.0f, ay = 0.0f;
        uint32_t node = 1;
        // LEARN: the warp's accepted cells not yet written out; lane j holds
        // the j-th of them
        int npend = 0;
        uint32_t my_cell = 0;
        if (LEARN) {
            // the group's centroid and second moments about it
            const float cnt = (float)__popc(__ballot_sync(kFull, active));
            float sx = active ? px : 0.0f, sy = active ? py : 0.0f;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                sx += __shfl_xor_sync(kFull, sx, o);
                sy += __shfl_xor_sync(kFull, sy, o);
            }
            const float gx = sx / cnt, gy = sy / cnt;
            const float u = active ? px - gx : 0.0f, v = active ? py - gy : 0.0f;
            float t0 = u * u + v * v, t1 = u * u - v * v, t2 = 2.0f * u * v;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                t0 += __shfl_xor_sync(kFull, t0, o);
                t1 += __shfl_xor_sync(kFull, t1, o);
                t2 += __shfl_xor_sync(kFull, t2, o);
            }
            if (lane == 0) {
                lb.ggeo[2 * w] = make_float4(gx, gy, t0 / cnt, cnt);
                lb.ggeo[2 * w + 1] = make_float4(t1 / cnt, t2 / cnt, 0.0f, 0.0f);
            }
        }
        // LEARN: the pending cells the group sees at a size ratio h / d of at
        // least kLearnMinRatio theta (d from the group's centroid) to this
        // warp's segment of the pair list, one atomic per flush
        auto flush = [&]() {
            __syncwarp();  // lane 0's store of the centroid is seen by all lanes
            bool keep = false;
            if (lane < npend) {
                const float4 cell = __ldg(&nodes[my_cell]);
                const float4 g0 = lb.ggeo[2 * w];
                keep = learn_keep(s_dq[meta_level(__float_as_int(cell.w))], g0.x - cell.x,
                                  g0.y - cell.y, prm.epssq);
            }
            const unsigned km = __ballot_sync(kFull, keep);
            const unsigned nk = (unsigned)__popc(km);
            const uint32_t seg = (blockIdx.x * (kTravThreads / kWarp) + (threadIdx.x >> 5)) %
                                 (uint32_t)kPairSegments;
            uint32_t base = 0;
            if (lane == 0 && nk) base = atomicAdd(&ctr->pair_count[seg], nk);
            base = __shfl_sync(kFull, base, 0);
            const uint32_t idx = base + (uint32_t)__popc(km & ((1u << lane) - 1u));
            if (keep && idx < lb.seg_cap)
                lb.pairs[(size_t)seg * lb.seg_cap + idx] = make_uint2((uint32_t)w, my_cell);
            if (lane == 0 && base + nk > lb.seg_cap) atomicOr(&st->err, kErrPairs);
            npend = 0;
        };
        // An opened cell's first child is node + 1 and always exists, so only
        // a jump to "next" can end the walk.
        if (!QUAD && node < end) {
            for (;;) {
                const float4 r = __ldg(&nodes[node]);
                const int meta = __float_as_int(r.w);
                const float dx = px - r.x, dy = py - r.y;
                const float d2 = sq_dist(dx, dy, prm.epssq);
                // written as !(d2 < dq): a NaN distance accepts, so a warp
                // with a non-finite lane still ends its walk
                if (__all_sync(kFull, !(d2 < s_dq[meta_level(meta)]))) {
                    float c;
                    if (OVERLAP && meta_level(meta) == kBodyLevel)
                        c = overlap_factor(d2, my_size, ssize[owner[node] >> 6], r.z);
                    else
                        c = __fdividef(r.z, d2);
                    ax = fmaf(dx, c, ax);
                    ay = fmaf(dy, c, ay);
                    if (LEARN && meta_level(meta) != kBodyLevel) {
                        if (lane == npend) my_cell = node;
                        if (++npend == 32) flush();
                    }
                    node = meta_next(meta);
                    if (node >= end) break;
                } else {
                    ++node;
                }
            }
        }
        if (QUAD && node < end) {
            float4 r = __ldg(&nodes[node]);
            for (;;) {
                const int meta = __float_as_int(r.w);
                const int lvl = meta_level(meta);
                const float m = r.z;
                const float dx = px - r.x, dy = py - r.y;
                const float d2 = sq_dist(dx, dy, prm.epssq);
                if (__all_sync(kFull, !(d2 < s_dq[lvl]))) {
                    const uint32_t next = meta_next(meta);
                    // the loads of the next node (and of this cell's second
                    // moment) go out before this node's sums, so the warp
                    // does not wait on them one after the other
                    float2 q = make_float2(0.0f, 0.0f);
                    if (lvl != kBodyLevel) q = __ldg(&quad[node]);
                    if (next < end) r = __ldg(&nodes[next]);
                    const float inv = __fdividef(1.0f, d2);
                    const float c = m * inv;
                    ax = fmaf(dx, c, ax);
                    ay = fmaf(dy, c, ay);
                    if (lvl != kBodyLevel) {
                        // conj(a2) u^3 with u = 1 / conj(w) = w / |w|^2: |u| <= 1 / sqrt(eps)
                        // and |a2 u^3| is below the monopole term's size, so nothing
                        // overflows however far apart the bodies are
                        const float ux = dx * inv, uy = dy * inv;
                        const float xx = ux * ux, yy = uy * uy;
                        const float ur = ux * fmaf(-3.0f, yy, xx);
                        const float ui = uy * fmaf(-3.0f, xx, yy);
                        ax = fmaf(q.x, ur, fmaf(-q.y, ui, ax));
                        ay = fmaf(-q.x, ui, fmaf(-q.y, ur, ay));
                        if (LEARN) {
                            if (lane == npend) my_cell = node;
                            if (++npend == 32) flush();
                        }
                    }
                    node = next;
                    if (node >= end) break;
                } else {
                    ++node;
                    r = __ldg(&nodes[node]);
                }
            }
        }
        // rounded on its own (never fused into the force sum that follows), so
        // the learned iteration, which stores it, adds the same value
        const float kmi = prm.k_r * me.z;
        ax = __fmul_rn(ax, kmi);
        ay = __fmul_rn(ay, kmi);
        if (LEARN) {
            if (npend) flush();
            if (active) lb.rep[k] = make_float2(ax, ay);
            continue;
        }
        float sw = 0.0f, tr = 0.0f;
        if (active) {
            const uint32_t i = vals[k];
            const float2 g = fag[i], fp = fprev[i];
            const float fx = g.x + ax, fy = g.y + ay;
            f[i] = make_float2(fx, fy);
            float dx = fx - fp.x, dy = fy - fp.y;
            sw = me.z * sqrtf(sq_norm(dx, dy));
            dx = fx + fp.x;
            dy = fy + fp.y;
            tr = me.z * (float)(sqrtf(sq_norm(dx, dy)) / 2.0);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            sw += __shfl_xor_sync(kFull, sw, o);
            tr += __shfl_xor_sync(kFull, tr, o);
        }
        if (lane == 0) warp_partial[w] = make_float2(sw, tr);
    }
    if (LEARN) return;
    // last block: fixed-order sum of the per-warp partials, then the speed rule
    speed_finish<kTravThreads>(n, warp_partial, &ctr->trav_done, st, s_last, s_red);
}

// The walk of k_traverse without the force arithmetic, over the tree still in
// the node array (the last step's), with the root radius that step used:
// counts its body-node interactions and acceptance tests.  Diagnostics only;
// the stepping path does not launch it.
__global__ void __launch_bounds__(kTravThreads) k_count_interactions(
    int n, const float4 *__restrict nodes, const uint32_t *__restrict body_node, DevState *st,
    Params prm) {
    __shared__ float s_dq[64];
    // no tree yet, or the last step stopped before its tree was complete
    if (st->err || st->poison || st->tree_nodes == 0) return;
    if (threadIdx.x == 0) {
        float tmp = st->trav_radius * 2;
        float dq = tmp * tmp * prm.itolsq;
        s_dq[0] = 0.0f;
        for (int l = 1; l <= kLevels; ++l) {
            s_dq[l] = dq + prm.epssq;
            dq = dq * 0.25f;
        }
        for (int l = kLevels + 1; l < 64; ++l) s_dq[l] = 0.0f;
    }
    __syncthreads();
    const uint32_t end = st->tree_nodes;
    const int lane = threadIdx.x & 31;
    const int nwarps = (n + 31) >> 5;
    const int stride = (int)(gridDim.x * blockDim.x) >> 5;
    for (int w = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); w < nwarps; w += stride) {
        const int k = w * 32 + lane;
        const bool active = k < n;
        const float4 me = nodes[body_node[active ? k : n - 1]];
        const float px = active ? me.x : 1e30f, py = active ? me.y : 1e30f;
        unsigned long long acc = 0, steps = 0;
        uint32_t node = 1;
        while (node < end) {
            const float4 r = nodes[node];
            const int meta = __float_as_int(r.w);
            const float dx = px - r.x, dy = py - r.y;
            const float d2 = sq_dist(dx, dy, prm.epssq);
            ++steps;
            if (__all_sync(kFull, !(d2 < s_dq[meta_level(meta)]))) {
                ++acc;
                node = meta_next(meta);
            } else {
                ++node;
            }
        }
        if (lane == 0) {
            const unsigned long long lanes = (unsigned long long)min(32, n - w * 32);
            atomicAdd(&st->interactions, acc * lanes);
            atomicAdd(&st->visits, steps * lanes);
        }
    }
}

// --------------------------------------------------------------- displace --

// DisplacementKernel (src/RPFA2Kernels.cu:223-251), fused with the bounding
// box of the new positions, which the next iteration's tree needs
// (BoundingBoxKernel, src/RPBHKernels.cu:70-157).
// ------------------------------------------------------------ exact f64 --

// The exact all-pairs repulsion of a few sampled bodies in double precision,
// the yardstick for the tree's approximation error: one block per sampled
// body i (an internal id), out[s] = k_r m_i sum_{j != i} m_j d / (d^2 + eps),
// d = p_i - p_j.  Each thread sums a fixed stride of j and the block reduces
// in a fixed order, so the result does not depend on timing.
constexpr int kExactThreads = 256;

__global__ void __launch_bounds__(kExactThreads) k_exact_f64(int n, const float2 *__restrict pos,
                                                             const float *__restrict mass,
                                                             const uint32_t *__restrict ids,
                                                             double2 *__restrict out, Params prm) {
    __shared__ double s_x[kExactThreads], s_y[kExactThreads];
    const uint32_t i = ids[blockIdx.x];
    double ax = 0.0, ay = 0.0;
    if (i < (uint32_t)n) {
        const double px = pos[i].x, py = pos[i].y;
        for (int j = threadIdx.x; j < n; j += kExactThreads) {
            if ((uint32_t)j == i) continue;
            const double dx = px - pos[j].x, dy = py - pos[j].y;
            const double c = (double)mass[j] / (dx * dx + dy * dy + (double)prm.epssq);
            ax += dx * c;
            ay += dy * c;
        }
    }
    s_x[threadIdx.x] = ax;
    s_y[threadIdx.x] = ay;
    __syncthreads();
    for (int o = kExactThreads / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            s_x[threadIdx.x] += s_x[threadIdx.x + o];
            s_y[threadIdx.x] += s_y[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double kmi = i < (uint32_t)n ? (double)prm.k_r * mass[i] : 0.0;
        out[blockIdx.x] = make_double2(kmi * s_x[0], kmi * s_y[0]);
    }
}

// ------------------------------------------------------------------ guard --

// The accuracy guard's three views of the repulsion of ns sampled sorted
// bodies (k = (2s + 1) n / 2ns), all from the last iteration's tree, whose
// body records hold the positions that iteration used:
//   exact  k_r m_k sum_{j != k} m_j d / (d^2 + eps) over every body, FP64;
//   plain  the reference walk (monopole, theta = 1) of the sample's own group
//          of 32 sorted bodies over that tree;
//   cur    what the iteration applied: its total force less gravity and
//          attraction.
__device__ __forceinline__ int guard_sample(int s, int ns, int n) {
    return (int)(((long long)(2 * s + 1) * n) / (2ll * ns));
}

// The exact sums are split over kGuardSplit blocks per sample (blockIdx.y
// takes a slice of the sorted bodies), so that the few hundred samples of a
// check fill the GPU; k_guard_finish adds the slices in a fixed order.
constexpr int kGuardSplit = 16;

__global__ void __launch_bounds__(kExactThreads) k_guard_exact(
    int n, int ns, const float4 *__restrict nodes, const uint32_t *__restrict body_node,
    Params prm, double2 *__restrict part) {
    __shared__ double s_x[kExactThreads], s_y[kExactThreads];
    const int k = guard_sample(blockIdx.x, ns, n);
    const float4 me = nodes[body_node[k]];
    const double px = me.x, py = me.y;
    const int per = (n + kGuardSplit - 1) / kGuardSplit;
    const int j0 = (int)blockIdx.y * per, j1 = min(n, j0 + per);
    double ax = 0.0, ay = 0.0;
    for (int j = j0 + threadIdx.x; j < j1; j += kExactThreads) {
        if (j == k) continue;
        const float4 o = nodes[body_node[j]];
        const double dx = px - o.x, dy = py - o.y;
        const double c = (double)o.z / (dx * dx + dy * dy + (double)prm.epssq);
        ax += dx * c;
        ay += dy * c;
    }
    s_x[threadIdx.x] = ax;
    s_y[threadIdx.x] = ay;
    __syncthreads();
    for (int o = kExactThreads / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            s_x[threadIdx.x] += s_x[threadIdx.x + o];
            s_y[threadIdx.x] += s_y[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0)
        part[(size_t)blockIdx.x * kGuardSplit + blockIdx.y] = make_double2(s_x[0], s_y[0]);
}

// One thread per sample: its slices' sums in order, times k_r m_i, and the
// repulsion the iteration applied to it.
__global__ void __launch_bounds__(256) k_guard_finish(
    int n, int ns, const float4 *__restrict nodes, const uint32_t *__restrict body_node,
    const uint32_t *__restrict vals, const float2 *__restrict f, const float2 *__restrict fag,
    Params prm, const double2 *__restrict part, double2 *__restrict exact,
    float2 *__restrict cur) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= ns) return;
    const int k = guard_sample(s, ns, n);
    double sx = 0.0, sy = 0.0;
    for (int c = 0; c < kGuardSplit; ++c) {
        const double2 v = part[(size_t)s * kGuardSplit + c];
        sx += v.x;
        sy += v.y;
    }
    const double kmi = (double)prm.k_r * nodes[body_node[k]].z;
    exact[s] = make_double2(kmi * sx, kmi * sy);
    const uint32_t i = vals[k];
    cur[s] = make_float2(f[i].x - fag[i].x, f[i].y - fag[i].y);
}

// One warp per sample: the plain walk of the sample's group (the k_traverse
// loop at theta = 1); the sample's lane keeps its sum.
__global__ void __launch_bounds__(256) k_guard_plain(int n, int ns,
                                                     const float4 *__restrict nodes,
                                                     const uint32_t *__restrict body_node,
                                                     const DevState *st, Params prm,
                                                     float2 *__restrict plain) {
    __shared__ float s_dq[64];
    if (threadIdx.x == 0) {
        // the thresholds of k_traverse for theta = 1, from the radius that
        // iteration's walk used
        float tmp = st->trav_radius * 2;
        float dq = tmp * tmp * 1.0f;
        s_dq[0] = 0.0f;
        for (int l = 1; l <= kLevels; ++l) {
            s_dq[l] = dq + prm.epssq;
            dq = dq * 0.25f;
        }
        for (int l = kLevels + 1; l < 64; ++l) s_dq[l] = 0.0f;
    }
    __syncthreads();
    const int s = blockIdx.x * (256 / kWarp) + (threadIdx.x >> 5);
    if (s >= ns) return;
    const int lane = threadIdx.x & 31;
    const int ks = guard_sample(s, ns, n);
    const int k = (ks & ~31) + lane;
    const bool active = k < n;
    const float4 me = nodes[body_node[active ? k : n - 1]];
    const float px = active ? me.x : 1e30f, py = active ? me.y : 1e30f;
    const uint32_t end = st->tree_nodes;
    float ax = 0.0f, ay = 0.0f;
    uint32_t node = 1;
    if (node < end) {
        for (;;) {
            const float4 r = __ldg(&nodes[node]);
            const int meta = __float_as_int(r.w);
            const float dx = px - r.x, dy = py - r.y;
            const float d2 = sq_dist(dx, dy, prm.epssq);
            if (__all_sync(kFull, !(d2 < s_dq[meta_level(meta)]))) {
                const float c = __fdividef(r.z, d2);
                ax = fmaf(dx, c, ax);
                ay = fmaf(dy, c, ay);
                node = meta_next(meta);
                if (node >= end) break;
            } else {
                ++node;
            }
        }
    }
    if (k == ks) {
        const float kmi = prm.k_r * me.z;
        plain[s] = make_float2(ax * kmi, ay * kmi);
    }
}

// 4 blocks per SM (32 registers): the launch's up to 4 blocks per SM are all
// resident at once
__global__ void __launch_bounds__(kDispThreads, 2048 / kDispThreads) k_displace(int n, float2 *__restrict pos,
                                                           const float2 *__restrict f,
                                                           float2 *__restrict fprev,
                                                           float4 *__restrict partial, DevState *st,
                                                           IterCounters *ctr) {
    if (st->err || st->poison) return;
    const float global_speed = st->global_speed;
    float4 a = make_float4(FLT_MAX, -FLT_MAX, FLT_MAX, -FLT_MAX);
    bool bad = false;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float2 fi = f[i], fp = fprev[i];
        const float factor = displacement_factor(fi, fp, global_speed);
        float2 p = pos[i];
        p.x += fi.x * factor;
        p.y += fi.y * factor;
        pos[i] = p;
        fprev[i] = fi;
        a = bbox_merge(a, make_float4(p.x, p.x, p.y, p.y));
        bad |= !(isfinite(p.x) && isfinite(p.y));
    }
    bbox_finish<kDispThreads>(a, bad, partial, &ctr->disp_done, st);
    if (blockIdx.x == 0 && threadIdx.x == 0) st->iters_done += 1;
}

// ---------------------------------------------------------------- attract --

// Gravity (GravityKernel, src/RPFA2Kernels.cu:35-73) plus attraction summed
// per node over its symmetric CSR row (AttractiveForceKernel :75-109 without
// atomics).  Rows hold neighbour ids padded with the row's own id to a
// multiple of four (a padding entry adds p_i - p_i = 0), so a lane loads four
// ids with one 16-byte load.  `lanes` lanes share a row and reduce with
// shuffles; heavy rows take a whole block.  To keep many loads in flight a
// warp of a short-row bucket works on kAttractBatch groups of rows at once:
// all column loads first, then all position gathers.  Neighbour-position
// gathers go through L1, which keeps the positions of the hubs (the first
// internal ids, gathered most often); a copy of the hubs in shared memory
// measured slower, its carve-out taking the L1 that the other gathers hit.
struct Gather {
    const float2 *__restrict pos;
    __device__ __forceinline__ float2 operator()(int c) const { return __ldg(&pos[c]); }
};

// Four neighbours of one CSR chunk.  WEIGHTED multiplies each pull by the
// edge's w^delta (edge weight influence, `delta` of src/RPForceAtlas2.hpp:49:
// f_a = w^delta d); a padding entry's pull is zero whatever its weight.  The
// products are rounded on their own, so a weight of 1 leaves the sums bit for
// bit those of the unweighted pass.
template <bool LINLOG, bool WEIGHTED>
__device__ __forceinline__ void add_four(const int4 c, const float4 w, const float2 p,
                                         const Gather &g, float &ax, float &ay) {
    float2 q0 = pull<LINLOG>(g(c.x), p), q1 = pull<LINLOG>(g(c.y), p);
    float2 q2 = pull<LINLOG>(g(c.z), p), q3 = pull<LINLOG>(g(c.w), p);
    if (WEIGHTED) {
        q0 = make_float2(__fmul_rn(q0.x, w.x), __fmul_rn(q0.y, w.x));
        q1 = make_float2(__fmul_rn(q1.x, w.y), __fmul_rn(q1.y, w.y));
        q2 = make_float2(__fmul_rn(q2.x, w.z), __fmul_rn(q2.y, w.z));
        q3 = make_float2(__fmul_rn(q3.x, w.w), __fmul_rn(q3.y, w.w));
    }
    ax += q0.x + q1.x + (q2.x + q3.x);
    ay += q0.y + q1.y + (q2.y + q3.y);
}

template <bool WEIGHTED>
__device__ __forceinline__ float4 chunk_weights(const float4 *__restrict w4, uint32_t q) {
    return WEIGHTED ? __ldcs(&w4[q]) : make_float4(1.0f, 1.0f, 1.0f, 1.0f);
}

// Rows of at most LANES int4 chunks (LANES <= 16): one chunk per lane.
template <int LANES, bool LINLOG, bool WEIGHTED>
__device__ __forceinline__ void attract_short_rows(int row0, int row_end, const Gather &g,
                                                   const float *__restrict mass,
                                                   const uint32_t *__restrict off,
                                                   const int4 *__restrict col4,
                                                   const float4 *__restrict w4,
                                                   float2 *__restrict fag, const Params &prm,
                                                   int lane) {
    constexpr int R = 32 / LANES;  // rows per warp and batch
    const int sub = lane / LANES, sl = lane % LANES;
    int row[kAttractBatch];
    bool has[kAttractBatch];
    int4 c[kAttractBatch];
    float4 w[kAttractBatch];
    float2 p[kAttractBatch];
#pragma unroll
    for (int u = 0; u < kAttractBatch; ++u) {
        row[u] = row0 + u * R + sub;
        const bool valid = row[u] < row_end;
        const uint32_t q = valid ? (off[row[u]] >> 2) + sl : 0u;
        const uint32_t e = valid ? off[row[u] + 1] >> 2 : 0u;
        has[u] = q < e;
        c[u] = has[u] ? __ldcs(&col4[q]) : make_int4(0, 0, 0, 0);
        w[u] = has[u] ? chunk_weights<WEIGHTED>(w4, q) : make_float4(1.0f, 1.0f, 1.0f, 1.0f);
        p[u] = valid ? g.pos[row[u]] : make_float2(0.0f, 0.0f);
    }
#pragma unroll
    for (int u = 0; u < kAttractBatch; ++u) {
        float ax = 0.0f, ay = 0.0f;
        if (has[u]) add_four<LINLOG, WEIGHTED>(c[u], w[u], p[u], g, ax, ay);
#pragma unroll
        for (int o = LANES / 2; o > 0; o >>= 1) {
            ax += __shfl_xor_sync(kFull, ax, o);
            ay += __shfl_xor_sync(kFull, ay, o);
        }
        if (row[u] < row_end && sl == 0)
            fag[row[u]] = with_gravity(p[u], mass[row[u]], ax, ay, prm);
    }
}

// Partial attraction of one row over chunks [b + first, e) with stride
// STRIDE, four chunks in flight per lane.
template <int STRIDE, bool LINLOG, bool WEIGHTED>
__device__ __forceinline__ void attract_long_row(uint32_t b, uint32_t e, int first, float2 p,
                                                 const Gather &g,
                                                 const int4 *__restrict col4,
                                                 const float4 *__restrict w4, float &ax,
                                                 float &ay) {
    uint32_t q = b + first;
    for (; q + 3 * STRIDE < e; q += 4 * STRIDE) {
        const int4 c0 = __ldcs(&col4[q]), c1 = __ldcs(&col4[q + STRIDE]);
        const int4 c2 = __ldcs(&col4[q + 2 * STRIDE]), c3 = __ldcs(&col4[q + 3 * STRIDE]);
        const float4 w0 = chunk_weights<WEIGHTED>(w4, q);
        const float4 w1 = chunk_weights<WEIGHTED>(w4, q + STRIDE);
        const float4 w2 = chunk_weights<WEIGHTED>(w4, q + 2 * STRIDE);
        const float4 w3 = chunk_weights<WEIGHTED>(w4, q + 3 * STRIDE);
        add_four<LINLOG, WEIGHTED>(c0, w0, p, g, ax, ay);
        add_four<LINLOG, WEIGHTED>(c1, w1, p, g, ax, ay);
        add_four<LINLOG, WEIGHTED>(c2, w2, p, g, ax, ay);
        add_four<LINLOG, WEIGHTED>(c3, w3, p, g, ax, ay);
    }
    for (; q < e; q += STRIDE)
        add_four<LINLOG, WEIGHTED>(__ldcs(&col4[q]), chunk_weights<WEIGHTED>(w4, q), p, g, ax,
                                   ay);
}

// The attraction pass: one block per work block of the plan (a row for the
// block-per-row bucket, 8 rows for the warp-per-row bucket, batches of short
// rows).
template <bool LINLOG, bool WEIGHTED>
__global__ void __launch_bounds__(256, (LINLOG || WEIGHTED) ? 4 : 8) k_attract(
    AttractPlan plan, const float2 *__restrict pos, const float *__restrict mass,
    const uint32_t *__restrict off, const int4 *__restrict col4, const float4 *__restrict w4,
    float2 *__restrict fag, Params prm) {
    __shared__ float2 s_red[256 / kWarp];
    const Gather g{pos};
    int bi = 0;
#pragma unroll 1
    for (int q = 1; q < plan.nbuckets; ++q)
        if ((int)blockIdx.x >= plan.b[q].block_begin) bi = q;
    const AttractBucket bk = plan.b[bi];
    const int blk = blockIdx.x - bk.block_begin;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (bk.lanes == 256) {
        // one row per block
        const int row = bk.row_begin + blk;
        const float2 p = g.pos[row];
        float ax = 0.0f, ay = 0.0f;
        attract_long_row<256, LINLOG, WEIGHTED>(off[row] >> 2, off[row + 1] >> 2, threadIdx.x, p,
                                                g, col4, w4, ax, ay);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            ax += __shfl_xor_sync(kFull, ax, o);
            ay += __shfl_xor_sync(kFull, ay, o);
        }
        if (lane == 0) s_red[wid] = make_float2(ax, ay);
        __syncthreads();
        if (threadIdx.x == 0) {
            ax = 0.0f;
            ay = 0.0f;
            for (int w = 0; w < 256 / kWarp; ++w) {
                ax += s_red[w].x;
                ay += s_red[w].y;
            }
            fag[row] = with_gravity(p, mass[row], ax, ay, prm);
        }
        return;
    }
    if (bk.lanes == 32) {
        // one row per warp
        const int row = bk.row_begin + blk * (256 / kWarp) + wid;
        if (row >= bk.row_end) return;
        const float2 p = g.pos[row];
        float ax = 0.0f, ay = 0.0f;
        attract_long_row<32, LINLOG, WEIGHTED>(off[row] >> 2, off[row + 1] >> 2, lane, p, g, col4,
                                               w4, ax, ay);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            ax += __shfl_xor_sync(kFull, ax, o);
            ay += __shfl_xor_sync(kFull, ay, o);
        }
        if (lane == 0) fag[row] = with_gravity(p, mass[row], ax, ay, prm);
        return;
    }
    // short rows: kAttractBatch groups of 32/lanes rows per warp
    const int row0 = bk.row_begin + (blk * (256 / kWarp) + wid) * kAttractBatch * (32 / bk.lanes);
    switch (bk.lanes) {
#define FA2_SHORT_ROWS(L) \
    attract_short_rows<L, LINLOG, WEIGHTED>(row0, bk.row_end, g, mass, off, col4, w4, fag, prm, lane)
        case 16: FA2_SHORT_ROWS(16); break;
        case 8: FA2_SHORT_ROWS(8); break;
        case 4: FA2_SHORT_ROWS(4); break;
        case 2: FA2_SHORT_ROWS(2); break;
        default: FA2_SHORT_ROWS(1); break;
#undef FA2_SHORT_ROWS
    }
}

// Gravity plus attraction with prevent_overlap: one warp per row of the
// padded CSR, each neighbour's pull (p_j - p_i) (d - s_i - s_j) / d while
// apart and nothing while overlapping (the paper's rule; a padding entry is
// the row's own id and pulls nothing), times w^delta with edge weights.
template <bool WEIGHTED>
__global__ void __launch_bounds__(256) k_attract_overlap(
    int n, const float2 *__restrict pos, const float *__restrict mass,
    const float *__restrict size, const uint32_t *__restrict off, const int *__restrict col,
    const float *__restrict wcol, float2 *__restrict fag, Params prm) {
    const int lane = threadIdx.x & 31;
    const int row = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (row >= n) return;
    const float2 p = pos[row];
    const float si = size[row];
    float ax = 0.0f, ay = 0.0f;
    for (uint32_t q = off[row] + lane; q < off[row + 1]; q += 32) {
        const int j = col[q];
        const float2 o = pos[j];
        const float dx = o.x - p.x, dy = o.y - p.y;
        const float d = sqrtf(dx * dx + dy * dy);
        const float dp = d - si - size[j];
        float w = dp > 0.0f ? dp / d : 0.0f;
        if (WEIGHTED) w *= wcol[q];
        ax = fmaf(dx, w, ax);
        ay = fmaf(dy, w, ay);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        ax += __shfl_xor_sync(kFull, ax, o);
        ay += __shfl_xor_sync(kFull, ay, o);
    }
    if (lane == 0) fag[row] = with_gravity(p, mass[row], ax, ay, prm);
}

__global__ void k_sorted_sizes(int n, const float *__restrict size,
                               const uint32_t *__restrict vals, float *__restrict ssize,
                               const DevState *st) {
    if (st->err || st->poison) return;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
        ssize[k] = size[vals[k]];
}

// ----------------------------------------------------------- permutations --

__global__ void k_scatter_xy(int n, const uint32_t *__restrict ref_of,
                             const float2 *__restrict src_ref, float2 *__restrict dst_int) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        dst_int[i] = src_ref[ref_of[i]];
}

__global__ void k_gather_xy(int n, const uint32_t *__restrict ref_of,
                            const float2 *__restrict src_int, float2 *__restrict dst_ref) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        dst_ref[ref_of[i]] = src_int[i];
}

__global__ void k_sorted_ref_ids(int n, const uint32_t *__restrict ref_of,
                                 const uint32_t *__restrict vals, uint32_t *__restrict out) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
        out[k] = ref_of[vals[k]];
}

inline int grid_for(int n, int threads, int cap) {
    int g = (n + threads - 1) / threads;
    return g < 1 ? 1 : (g > cap ? cap : g);
}

}  // namespace

// ---------------------------------------------------------------- launchers --

void launch_bbox(const Buffers &b, int nblocks, cudaStream_t s) {
    k_bbox<<<nblocks, kBBoxThreads, 0, s>>>(b.n, b.pos, b.bbox_partial, b.st, b.ctr);
}

void launch_keys(const Buffers &b, int nsm, cudaStream_t s) {
    (void)nsm;
    // the first sort pass reads buffer (first & 1), so the passes end in buffer 0
    const int in = b.sort_first & 1;
    k_keys<<<sort_tiles(b.n, b.sort_rounds), 1024, 0, s>>>(
        b.n, kSortThreads * b.sort_rounds, b.sort_first, b.pos, b.st, b.keys[in], b.vals[in],
        b.ctr, b.sort_counts);
}





void launch_traverse(const Buffers &b, const Params &p, int nblocks, cudaStream_t s) {
    const LearnBuffers none{};
    auto go = [&](auto kernel) {
        kernel<<<nblocks, kTravThreads, 0, s>>>(b.n, b.nodes, b.quad, b.body_node, b.vals[0],
                                                b.fag, b.fprev, b.f, b.warp_partial, b.st, b.ctr,
                                                p, none, nullptr, nullptr);
    };
    if (p.overlap) {
        k_traverse<false, false, true><<<nblocks, kTravThreads, 0, s>>>(
            b.n, b.nodes, b.quad, b.body_node, b.vals[0], b.fag, b.fprev, b.f, b.warp_partial,
            b.st, b.ctr, p, none, b.owner, b.ssize);
        return;
    }
    if (p.multipole >= 2)
        go(k_traverse<true, false>);
    else
        go(k_traverse<false, false>);
}

void launch_traverse_learn(const Buffers &b, const Params &p, const LearnBuffers &lb,
                           int nblocks, cudaStream_t s) {
    auto go = [&](auto kernel) {
        kernel<<<nblocks, kTravThreads, 0, s>>>(b.n, b.nodes, b.quad, b.body_node, b.vals[0],
                                                b.fag, b.fprev, b.f, b.warp_partial, b.st, b.ctr,
                                                p, lb, nullptr, nullptr);
    };
    if (p.multipole >= 2)
        go(k_traverse<true, true>);
    else
        go(k_traverse<false, true>);
}

size_t guard_part_count(int ns) { return (size_t)ns * kGuardSplit; }

void launch_guard(const Buffers &b, const Params &p, int ns, double2 *exact, float2 *plain,
                  float2 *cur, double2 *part, cudaStream_t s) {
    if (ns <= 0 || b.n <= 0) return;
    k_guard_exact<<<dim3(ns, kGuardSplit), kExactThreads, 0, s>>>(b.n, ns, b.nodes, b.body_node,
                                                                   p, part);
    k_guard_finish<<<(ns + 255) / 256, 256, 0, s>>>(b.n, ns, b.nodes, b.body_node, b.vals[0], b.f,
                                                    b.fag, p, part, exact, cur);
    k_guard_plain<<<(ns + 7) / 8, 256, 0, s>>>(b.n, ns, b.nodes, b.body_node, b.st, p, plain);
}

void launch_exact_f64(const Buffers &b, const Params &p, const uint32_t *ids, int n_ids,
                      double2 *out, cudaStream_t s) {
    if (n_ids <= 0) return;
    k_exact_f64<<<n_ids, kExactThreads, 0, s>>>(b.n, b.pos, b.mass, ids, out, p);
}

void launch_displace(const Buffers &b, int nsm, cudaStream_t s) {
    k_displace<<<grid_for(b.n, kDispThreads, nsm * 4), kDispThreads, 0, s>>>(
        b.n, b.pos, b.f, b.fprev, b.bbox_partial, b.st, b.ctr);
}

void launch_count_interactions(const Buffers &b, const Params &p, int nblocks, cudaStream_t s) {
    k_count_interactions<<<nblocks, kTravThreads, 0, s>>>(b.n, b.nodes, b.body_node, b.st, p);
}

void launch_attract(const Buffers &b, const Params &p, const AttractPlan &plan, cudaStream_t s) {
    if (plan.nblocks == 0) return;
    if (p.overlap) {
        const int blocks = (b.n + 7) / 8;
        const int *col = reinterpret_cast<const int *>(b.csr_col4);
        const float *w = reinterpret_cast<const float *>(b.csr_w4);
        if (w)
            k_attract_overlap<true><<<blocks, 256, 0, s>>>(b.n, b.pos, b.mass, b.size, b.csr_off,
                                                           col, w, b.fag, p);
        else
            k_attract_overlap<false><<<blocks, 256, 0, s>>>(b.n, b.pos, b.mass, b.size,
                                                            b.csr_off, col, w, b.fag, p);
        return;
    }
    const float4 *w4 = b.csr_w4;
    auto go = [&](auto kernel) {
        kernel<<<plan.nblocks, 256, 0, s>>>(plan, b.pos, b.mass, b.csr_off, b.csr_col4, w4, b.fag,
                                            p);
    };
    if (w4)
        p.linlog ? go(k_attract<true, true>) : go(k_attract<false, true>);
    else
        p.linlog ? go(k_attract<true, false>) : go(k_attract<false, false>);
}

void launch_sorted_sizes(const Buffers &b, cudaStream_t s) {
    k_sorted_sizes<<<grid_for(b.n, 256, 4096), 256, 0, s>>>(b.n, b.size, b.vals[0], b.ssize,
                                                            b.st);
}

void launch_scatter_xy(int n, const uint32_t *ref_of, const float2 *src_ref, float2 *dst_int,
                       cudaStream_t s) {
    k_scatter_xy<<<grid_for(n, 256, 4096), 256, 0, s>>>(n, ref_of, src_ref, dst_int);
}

void launch_gather_xy(int n, const uint32_t *ref_of, const float2 *src_int, float2 *dst_ref,
                      cudaStream_t s) {
    k_gather_xy<<<grid_for(n, 256, 4096), 256, 0, s>>>(n, ref_of, src_int, dst_ref);
}

void launch_sorted_ref_ids(int n, const uint32_t *ref_of, const uint32_t *vals, uint32_t *out,
                           cudaStream_t s) {
    k_sorted_ref_ids<<<grid_for(n, 256, 4096), 256, 0, s>>>(n, ref_of, vals, out);
}

int traverse_blocks_per_sm() {
    // the walk lives on L1 hits: give L1 the most of the SM's on-chip memory
    cudaFuncSetAttribute(k_traverse<false, false>, cudaFuncAttributePreferredSharedMemoryCarveout, 0);
    cudaFuncSetAttribute(k_traverse<true, false>, cudaFuncAttributePreferredSharedMemoryCarveout, 0);
    cudaFuncSetAttribute(k_traverse<false, false, true>,
                         cudaFuncAttributePreferredSharedMemoryCarveout, 0);
    // the learned walk keeps its pending pairs in registers, one per lane
    cudaFuncSetAttribute(k_traverse<false, true>, cudaFuncAttributePreferredSharedMemoryCarveout, 0);
    cudaFuncSetAttribute(k_traverse<true, true>, cudaFuncAttributePreferredSharedMemoryCarveout, 0);
    int nb = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_traverse<false, false>, kTravThreads, 0);
    return nb < 1 ? 1 : nb;
}

}  // namespace fa2
