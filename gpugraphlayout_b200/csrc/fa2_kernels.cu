// fa2_kernels.cu -- the per-iteration kernels of the B200 ForceAtlas2 engine
// except the radix sort (fa2_sort.cu).
//
// Quadtree.  The reference builds its quadtree by concurrent lock-based
// insertion (src/RPBHKernels.cu:184-329); the shape of that tree does not
// depend on insertion order: its cells are exactly the quadrant prefixes that
// hold at least two bodies.  Here the same tree is built without locks:
//   keys        each body's 32 quadrant digits, computed with the reference's
//               float cell-centre arithmetic and tie rule (:217-241), form a
//               64-bit Morton key;
//   sort        keys ascending = the reference's in-order body order (sortd);
//   runs        equal keys (only possible past depth 32) are ordered by
//               deeper digits; exactly coincident bodies are flagged;
//   tree_count  LCP of neighbouring keys (in quadrant digits) gives, per
//               body k, the cells that start at k: levels L[k-1]+1 .. L[k];
//               a scan gives every node its preorder index;
//   emit        writes each node once: position/mass of bodies, level and
//               subtree end of cells, parent links;
//   summarize   bottom-up mass and centre of mass, children in quadrant order
//               (SummarizationKernel :357-506), with the last child to finish
//               computing its parent instead of spin-waiting.
// The tree is stored in preorder with each node's "next" index (the node
// after its subtree), so the traversal needs no stack.
#include <float.h>
#include <stdint.h>

#include <cuda/atomic>

#include "fa2_internal.cuh"

namespace fa2 {

namespace {

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ int lcp_digits(uint64_t a, uint64_t b) {
    uint64_t x = a ^ b;
    return x == 0 ? kLevels : (__clzll(x) >> 1);
}

__device__ __forceinline__ int meta_level(int meta) { return meta & 63; }
__device__ __forceinline__ uint32_t meta_next(int meta) { return (uint32_t)meta >> kMetaShift; }
__device__ __forceinline__ float make_meta(uint32_t next, int level) {
    return __int_as_float((int)((next << kMetaShift) | (uint32_t)level));
}

// Quadrant digits of (px, py) under the root cell, computed the way
// TreeBuildingKernel walks down (src/RPBHKernels.cu:217-241): the child
// centre is the parent centre +/- r, r halving per level; a coordinate
// equal to the centre goes to the low side.
__device__ __forceinline__ uint64_t morton_key(float px, float py, float x, float y, float r) {
    uint64_t key = 0;
#pragma unroll 8
    for (int lvl = 0; lvl < kLevels; ++lvl) {
        r *= 0.5f;
        int j = 0;
        float dx = -r, dy = -r;
        if (x < px) {
            j = 1;
            dx = r;
        }
        if (y < py) {
            j |= 2;
            dy = r;
        }
        x = __fadd_rn(x, dx);
        y = __fadd_rn(y, dy);
        key = (key << 2) | (uint64_t)j;
    }
    return key;
}

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
// the block must call it.
template <int THREADS>
__device__ void bbox_finish(float4 a, float4 *__restrict partial, unsigned *done, DevState *st) {
    __shared__ float4 s_w[THREADS / kWarp];
    __shared__ bool s_last;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
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
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float2 p = pos[i];
        a = bbox_merge(a, make_float4(p.x, p.x, p.y, p.y));
    }
    bbox_finish<kBBoxThreads>(a, partial, &ctr->bbox_done, st);
}

// ------------------------------------------------------------------- keys --

// One block per sort tile: the tile's keys, the digit-0 counts of the tile
// (the first sort pass's per-tile input) and the tile's share of the digit
// histograms of all eight passes (order-independent, so counted once here).
__global__ void __launch_bounds__(256) k_keys(int n, const float2 *__restrict pos,
                                              const DevState *__restrict st,
                                              uint64_t *__restrict keys, uint32_t *__restrict vals,
                                              IterCounters *ctr, uint32_t *__restrict counts0) {
    __shared__ unsigned s_hist[8][256];
    if (st->err || st->poison) return;
    for (int j = threadIdx.x; j < 8 * 256; j += blockDim.x) (&s_hist[0][0])[j] = 0;
    __syncthreads();
    const float rx = st->rootx, ry = st->rooty, rr = st->radius;
    const int tile0 = blockIdx.x * kSortTile;
    const int tile_end = min(n, tile0 + kSortTile);
    for (int i = tile0 + threadIdx.x; i < tile_end; i += blockDim.x) {
        float2 p = pos[i];
        uint64_t key = morton_key(p.x, p.y, rx, ry, rr);
        keys[i] = key;
        vals[i] = (uint32_t)i;
#pragma unroll
        for (int ps = 0; ps < 8; ++ps) atomicAdd(&s_hist[ps][(key >> (8 * ps)) & 255], 1u);
    }
    __syncthreads();
    for (int j = threadIdx.x; j < 8 * 256; j += blockDim.x) {
        unsigned c = (&s_hist[0][0])[j];
        if (j < 256) counts0[(size_t)blockIdx.x * 256 + j] = c;
        if (c) atomicAdd(&(&ctr->hist[0][0])[j], c);
    }
}

// ------------------------------------------------------------------- runs --

// Replays the cell centre of a 32-digit key path.
__device__ __forceinline__ void key_centre(uint64_t key, float rx, float ry, float rr, float &x,
                                           float &y, float &r) {
    x = rx;
    y = ry;
    r = rr;
    for (int lvl = 0; lvl < kLevels; ++lvl) {
        r *= 0.5f;
        int j = (int)(key >> (2 * (kLevels - 1 - lvl))) & 3;
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
        int ja = (x < pa.x ? 1 : 0) | (y < pa.y ? 2 : 0);
        int jb = (x < pb.x ? 1 : 0) | (y < pb.y ? 2 : 0);
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

__global__ void __launch_bounds__(kCountThreads) k_tree_count(
    int n, const uint64_t *__restrict keys, int8_t *__restrict lcp, uint32_t *__restrict group,
    int32_t *__restrict cnt, int4 *__restrict kids, uint32_t capacity, DevState *st, IterCounters *ctr,
    uint32_t *status, uint32_t *__restrict vals, float2 *__restrict pos,
    const uint32_t *__restrict ref_of) {
    __shared__ int s_tile;
    __shared__ uint32_t s_warp[kCountThreads / kWarp];
    __shared__ uint32_t s_prefix;
    if (st->err || st->poison) return;
    if (threadIdx.x == 0) s_tile = atomicAdd(&ctr->count_ticket, 1u);
    __syncthreads();
    const int tile = s_tile;
    const int base = tile * kCountTile + threadIdx.x * kCountItems;
    int g[kCountItems];
    uint32_t sum = 0, run_starts = 0;
#pragma unroll
    for (int e = 0; e < kCountItems; ++e) {
        int k = base + e;
        g[e] = 0;
        if (k < n) {
            int Lk = lcp_at(keys, n, k);
            int Lkm1 = lcp_at(keys, n, k - 1);
            lcp[k] = (int8_t)Lk;
            g[e] = cells_at(k, Lk, Lkm1) + 1;
            // a run of equal 64-bit keys starts here (trees past depth 32)
            if (Lk == kLevels && Lkm1 != kLevels) run_starts |= 1u << e;
        }
        sum += (uint32_t)g[e];
    }
    // block exclusive scan of per-thread sums
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t inc = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(kFull, inc, o);
        if (lane >= o) inc += t;
    }
    if (lane == 31) s_warp[wid] = inc;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t run = 0;
        for (int w = 0; w < kCountThreads / kWarp; ++w) {
            uint32_t t = s_warp[w];
            s_warp[w] = run;
            run += t;
        }
        // decoupled look-back over tiles: flag in bit 31, value below
        const uint32_t kAgg = 1u << 30, kPre = 2u << 30, kMask = (1u << 30) - 1;
        uint32_t prefix = 0;
        if (tile == 0) {
            atomicExch(&status[0], kPre | run);
        } else {
            atomicExch(&status[tile], kAgg | run);
            int t = tile - 1;
            long spins = 0;
            while (t >= 0) {
                uint32_t s = *((volatile uint32_t *)&status[t]);
                if ((s >> 30) == 0) {
                    if (++spins > (1L << 22)) {
                        atomicOr(&st->err, kErrScanWait);
                        break;
                    }
                    continue;
                }
                prefix += s & kMask;
                if ((s >> 30) == 2) break;
                --t;
            }
            atomicExch(&status[tile], kPre | (prefix + run));
        }
        s_prefix = prefix;
    }
    __syncthreads();
    uint32_t off = s_prefix + s_warp[wid] + inc - sum;
#pragma unroll
    for (int e = 0; e < kCountItems; ++e) {
        int k = base + e;
        if (k < n) {
            group[k] = off;
            for (int q = 0; q < g[e]; ++q)
                if (off + q < capacity) {
                    cnt[off + q] = 0;
                    kids[off + q] = make_int4(-1, -1, -1, -1);
                }
            if (k == n - 1) {
                uint32_t total = off + (uint32_t)g[e];
                st->tree_nodes = total;
                st->max_level = 0;  // raised by k_emit
                st->interactions = 0;  // counted by k_traverse
                st->visits = 0;
                if (total > capacity) atomicOr(&st->err, kErrTreeTooLarge);
            }
        }
        off += (uint32_t)g[e];
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
    int Lb = load_lcp(lcp, n, b), Lbm1 = load_lcp(lcp, n, b - 1);
    return group[b] + (uint32_t)cells_at(b, Lb, Lbm1);
}

// Index of the cell at level lam that contains sorted body k, given that it
// starts before k: its first body a is the smallest j with LCP(K_j, K_k) >= lam.
__device__ uint32_t find_cell(const uint64_t *__restrict keys, const int8_t *__restrict lcp,
                              const uint32_t *__restrict group, int n, int k, int lam) {
    const uint64_t kk = keys[k];
    int ok = k - 1;  // known to satisfy
    int step = 1, bad = -1;
    for (;;) {
        int j = ok - step;
        if (j < 0) {
            bad = -1;
            break;
        }
        if (lcp_digits(keys[j], kk) >= lam) {
            ok = j;
            step <<= 1;
        } else {
            bad = j;
            break;
        }
    }
    // smallest satisfying index in (bad, ok]
    int lo = bad + 1, hi = ok;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (lcp_digits(keys[mid], kk) >= lam)
            hi = mid;
        else
            lo = mid + 1;
    }
    const int a = lo;
    const int lo_level = a == 0 ? 0 : load_lcp(lcp, n, a - 1) + 1;
    return group[a] + (uint32_t)(lam - lo_level);
}

// Largest j >= k with LCP(K_k, K_j) >= lvl (the last body of the cell at
// level lvl that starts at k).
__device__ int find_end(const uint64_t *__restrict keys, int n, int k, int lvl) {
    const uint64_t kk = keys[k];
    int ok = k, step = 1, bad = n;
    for (;;) {
        int j = ok + step;
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
    int lo = ok, hi = bad - 1;  // largest satisfying in [ok, bad)
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (lcp_digits(keys[mid], kk) >= lvl)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

__global__ void __launch_bounds__(256) k_emit(int n, const uint64_t *__restrict keys,
                                              const uint32_t *__restrict vals,
                                              const int8_t *__restrict lcp,
                                              const uint32_t *__restrict group,
                                              const float2 *__restrict pos,
                                              const float *__restrict mass, float4 *__restrict nodes,
                                              int32_t *__restrict parent, int32_t *__restrict cnt,
                                              int4 *__restrict kids,
                                              uint32_t *__restrict body_node, DevState *st) {
    if (st->err || st->poison) return;
    int local_max = 0;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int Lk = load_lcp(lcp, n, k), Lkm1 = load_lcp(lcp, n, k - 1);
        const int c = cells_at(k, Lk, Lkm1);
        const uint32_t Gk = group[k];
        const uint32_t bnode = Gk + (uint32_t)c;
        const int lo_level = k == 0 ? 0 : Lkm1 + 1;
        // the body
        const uint32_t i = vals[k];
        const float2 p = pos[i];
        nodes[bnode] = make_float4(p.x, p.y, mass[i], make_meta(bnode + 1, kBodyLevel));
        body_node[k] = bnode;
        const int lam = max(max(Lk, Lkm1), 0);
        const uint32_t pb = c > 0 ? bnode - 1 : find_cell(keys, lcp, group, n, k, lam);
        parent[bnode] = (int32_t)pb;
        {
            const int slot = atomicAdd(&cnt[pb], 1);
            if (slot < 4) reinterpret_cast<int *>(kids)[4 * (size_t)pb + slot] = (int)bnode;
        }
        // the cells that start here, outermost first
        for (int q = 0; q < c; ++q) {
            const int lvl = lo_level + q;
            const uint32_t node = Gk + (uint32_t)q;
            const int b = lvl == 0 ? n - 1 : find_end(keys, n, k, lvl);
            const uint32_t next = body_index(lcp, group, n, b) + 1;
            nodes[node] = make_float4(0.0f, 0.0f, 0.0f, make_meta(next, lvl));
            int32_t par = -1;
            if (q > 0)
                par = (int32_t)node - 1;
            else if (lvl > 0)
                par = (int32_t)find_cell(keys, lcp, group, n, k, lvl - 1);
            parent[node] = par;
            if (par >= 0) {
                const int slot = atomicAdd(&cnt[par], 1);
                if (slot < 4) reinterpret_cast<int *>(kids)[4 * (size_t)par + slot] = (int)node;
            }
            local_max = max(local_max, lvl);
        }
    }
    local_max = __reduce_max_sync(kFull, local_max);
    if ((threadIdx.x & 31) == 0 && local_max > 0) atomicMax(&st->max_level, local_max);
}

// -------------------------------------------------------------- summarize --

__device__ __forceinline__ void cswap(uint32_t &a, uint32_t &b) {
    const uint32_t lo = min(a, b), hi = max(a, b);
    a = lo;
    b = hi;
}

__device__ __forceinline__ void add_child(const float4 &r, float &cm, float &px, float &py) {
    const float m = r.z;
    px += r.x * m;
    py += r.y * m;
    cm += m;
}

// Bottom-up cell mass and centre of mass.  Every node decrements its
// parent's child counter (acquire-release, so the last child sees what the
// others wrote); the child that brings it to zero computes the parent from
// all its children, in quadrant order, as SummarizationKernel does
// (src/RPBHKernels.cu:461-494), and continues upwards.  A cell's children
// come from the four slots k_emit filled; preorder index order is quadrant
// order.  Level-32 cells can hold more bodies than four slots and are
// walked through their next links instead.
__global__ void __launch_bounds__(256) k_summarize(int n, const uint32_t *__restrict body_node,
                                                   const int32_t *__restrict parent,
                                                   int32_t *cnt, const int4 *__restrict kids,
                                                   float4 *nodes, DevState *st) {
    if (st->err || st->poison) return;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        int32_t p = parent[body_node[k]];
        // a body publishes nothing (k_emit wrote it): relaxed arrival
        bool last = atomicSub(&cnt[p], 1) == 1;
        while (last) {
            cuda::atomic_thread_fence(cuda::memory_order_acquire, cuda::thread_scope_device);
            const float4 prec = __ldcg(&nodes[p]);
            const int32_t gp = __ldcg(&parent[p]);
            const int meta = __float_as_int(prec.w);
            float cm = 0.0f, px = 0.0f, py = 0.0f;
            if (meta_level(meta) == kLevels) {
                const uint32_t end = meta_next(meta);
                for (uint32_t c = (uint32_t)p + 1; c < end;) {
                    const float4 r = __ldcg(&nodes[c]);
                    add_child(r, cm, px, py);
                    c = meta_next(__float_as_int(r.w));
                }
            } else {
                const int4 kd = __ldcg(&kids[p]);
                uint32_t c0 = (uint32_t)kd.x, c1 = (uint32_t)kd.y, c2 = (uint32_t)kd.z,
                         c3 = (uint32_t)kd.w;  // empty slots are -1: sorted last
                cswap(c0, c1);
                cswap(c2, c3);
                cswap(c0, c2);
                cswap(c1, c3);
                cswap(c1, c2);
                const float4 r0 = __ldcg(&nodes[c0]);
                const float4 r1 = c1 != ~0u ? __ldcg(&nodes[c1]) : make_float4(0, 0, 0, 0);
                const float4 r2 = c2 != ~0u ? __ldcg(&nodes[c2]) : make_float4(0, 0, 0, 0);
                const float4 r3 = c3 != ~0u ? __ldcg(&nodes[c3]) : make_float4(0, 0, 0, 0);
                add_child(r0, cm, px, py);
                if (c1 != ~0u) add_child(r1, cm, px, py);
                if (c2 != ~0u) add_child(r2, cm, px, py);
                if (c3 != ~0u) add_child(r3, cm, px, py);
            }
            const float inv = 1.0f / cm;
            __stcg(&nodes[p], make_float4(px * inv, py * inv, cm, prec.w));
            if (gp < 0) break;
            // a cell publishes its summary to whoever completes its parent
            cuda::atomic_ref<int32_t, cuda::thread_scope_device> arrivals(cnt[gp]);
            last = arrivals.fetch_sub(1, cuda::memory_order_release) == 1;
            p = gp;
        }
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
__global__ void __launch_bounds__(kTravThreads, 2048 / kTravThreads) k_traverse(
    int n, const float4 *__restrict nodes, const uint32_t *__restrict body_node,
    const uint32_t *__restrict vals, const float2 *__restrict fag,
    const float2 *__restrict fprev, float2 *__restrict f, float2 *__restrict warp_partial,
    DevState *st, IterCounters *ctr, Params prm) {
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
    }
    __syncthreads();
    const uint32_t end = st->tree_nodes;
    const int lane = threadIdx.x & 31;
    const int nwarps = (n + 31) >> 5;
    // Groups of 32 bodies are handed out one at a time (the work per group
    // varies with the local density of the layout).
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
        const float kmi = prm.k_r * me.z;
        float ax = 0.0f, ay = 0.0f;
        uint32_t node = 1, n_acc = 0;
        while (node < end) {
            const float4 r = __ldg(&nodes[node]);
            const int meta = __float_as_int(r.w);
            const float dx = px - r.x, dy = py - r.y;
            const float d2 = dx * dx + dy * dy + prm.epssq;
            if (__all_sync(kFull, d2 >= s_dq[meta_level(meta)])) {
                const float c = __fdividef(kmi * r.z, d2);
                ax = fmaf(dx, c, ax);
                ay = fmaf(dy, c, ay);
                node = meta_next(meta);
                ++n_acc;
            } else {
                ++node;
            }
        }
        if (lane == 0) {
            const unsigned lanes = (unsigned)min(32, n - w * 32);
            atomicAdd(&st->interactions, (unsigned long long)n_acc * lanes);
        }
        float sw = 0.0f, tr = 0.0f;
        if (active) {
            const uint32_t i = vals[k];
            const float2 g = fag[i], fp = fprev[i];
            const float fx = g.x + ax, fy = g.y + ay;
            f[i] = make_float2(fx, fy);
            float dx = fx - fp.x, dy = fy - fp.y;
            sw = me.z * sqrtf(dx * dx + dy * dy);
            dx = fx + fp.x;
            dy = fy + fp.y;
            tr = me.z * (float)(sqrtf(dx * dx + dy * dy) / 2.0);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            sw += __shfl_xor_sync(kFull, sw, o);
            tr += __shfl_xor_sync(kFull, tr, o);
        }
        if (lane == 0) warp_partial[w] = make_float2(sw, tr);
    }
    // last block: fixed-order sum of the per-warp partials, then the speed rule
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = atomicAdd(&ctr->trav_done, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    float sw = 0.0f, tr = 0.0f;
    for (int w = threadIdx.x; w < nwarps; w += blockDim.x) {
        float2 v = __ldcg(&warp_partial[w]);
        sw += v.x;
        tr += v.y;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        sw += __shfl_xor_sync(kFull, sw, o);
        tr += __shfl_xor_sync(kFull, tr, o);
    }
    if (lane == 0) {
        s_red[0][threadIdx.x >> 5] = sw;
        s_red[1][threadIdx.x >> 5] = tr;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        float swg = 0.0f, etra = 0.0f;
        for (int w = 0; w < kTravThreads / kWarp; ++w) {
            swg += s_red[0][w];
            etra += s_red[1][w];
        }
        st->swg_sum = swg;
        st->etra_sum = etra;
        // src/RPFA2Kernels.cu:243-275
        float estimated_optimal_jitter_tollerance = 0.05 * sqrtf((float)n);
        float minJT = sqrtf(estimated_optimal_jitter_tollerance);
        float jt = st->jitter_tolerance *
                   fmaxf(minJT, fminf(st->k_s_max, estimated_optimal_jitter_tollerance * etra /
                                                       powf((float)n, 2.0f)));
        float min_speed_efficiency = 0.05f;
        float se = st->speed_efficiency, gs = st->global_speed;
        if (swg / etra > 2.0) {
            if (se > min_speed_efficiency) se *= 0.5;
            jt = fmaxf(jt, st->jitter_tolerance);
        }
        float targetSpeed = jt * se * etra / swg;
        if (swg > jt * etra) {
            if (se > min_speed_efficiency) se *= 0.7;
        } else if (gs < 1000) {
            se *= 1.3;
        }
        float max_rise = 0.5f;
        gs += fminf(targetSpeed - gs, max_rise * gs);
        st->speed_efficiency = se;
        st->global_speed = gs;
    }
}

// --------------------------------------------------------------- displace --

// DisplacementKernel (src/RPFA2Kernels.cu:223-251), fused with the bounding
// box of the new positions, which the next iteration's tree needs
// (BoundingBoxKernel, src/RPBHKernels.cu:70-157).
__global__ void __launch_bounds__(kDispThreads) k_displace(int n, float2 *__restrict pos,
                                                           const float2 *__restrict f,
                                                           float2 *__restrict fprev,
                                                           float4 *__restrict partial, DevState *st,
                                                           IterCounters *ctr) {
    if (st->err || st->poison) return;
    const float global_speed = st->global_speed;
    float4 a = make_float4(FLT_MAX, -FLT_MAX, FLT_MAX, -FLT_MAX);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float2 fi = f[i], fp = fprev[i];
        const float dx = fi.x - fp.x, dy = fi.y - fp.y;
        const float swg = sqrtf(dx * dx + dy * dy);
        const float factor = global_speed / (1.0 + sqrtf(global_speed * swg));
        float2 p = pos[i];
        p.x += fi.x * factor;
        p.y += fi.y * factor;
        pos[i] = p;
        fprev[i] = fi;
        a = bbox_merge(a, make_float4(p.x, p.x, p.y, p.y));
    }
    bbox_finish<kDispThreads>(a, partial, &ctr->disp_done, st);
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
// all column loads first, then all position gathers.
__device__ __forceinline__ void add_four(const int4 c, const float2 p,
                                         const float2 *__restrict pos, float &ax, float &ay) {
    const float2 q0 = __ldg(&pos[c.x]), q1 = __ldg(&pos[c.y]);
    const float2 q2 = __ldg(&pos[c.z]), q3 = __ldg(&pos[c.w]);
    ax += (q0.x - p.x) + (q1.x - p.x) + ((q2.x - p.x) + (q3.x - p.x));
    ay += (q0.y - p.y) + (q1.y - p.y) + ((q2.y - p.y) + (q3.y - p.y));
}

__device__ __forceinline__ float2 with_gravity(float2 p, float m, float ax, float ay,
                                               const Params &prm) {
    float f_g;
    if (prm.strong_gravity)
        f_g = prm.k_g * m;
    else if (p.x != 0.0f || p.y != 0.0f)
        f_g = prm.k_g * m * rsqrtf(p.x * p.x + p.y * p.y);
    else
        f_g = 0.0f;
    return make_float2(-p.x * f_g + ax, -p.y * f_g + ay);
}

// Rows of at most LANES int4 chunks (LANES <= 16): one chunk per lane.
template <int LANES>
__device__ __forceinline__ void attract_short_rows(int row0, int row_end,
                                                   const float2 *__restrict pos,
                                                   const float *__restrict mass,
                                                   const uint32_t *__restrict off,
                                                   const int4 *__restrict col4,
                                                   float2 *__restrict fag, const Params &prm,
                                                   int lane) {
    constexpr int R = 32 / LANES;  // rows per warp and batch
    const int sub = lane / LANES, sl = lane % LANES;
    int row[kAttractBatch];
    bool has[kAttractBatch];
    int4 c[kAttractBatch];
    float2 p[kAttractBatch];
#pragma unroll
    for (int u = 0; u < kAttractBatch; ++u) {
        row[u] = row0 + u * R + sub;
        const bool valid = row[u] < row_end;
        const uint32_t q = valid ? (off[row[u]] >> 2) + sl : 0u;
        const uint32_t e = valid ? off[row[u] + 1] >> 2 : 0u;
        has[u] = q < e;
        c[u] = has[u] ? __ldcs(&col4[q]) : make_int4(0, 0, 0, 0);
        p[u] = valid ? pos[row[u]] : make_float2(0.0f, 0.0f);
    }
#pragma unroll
    for (int u = 0; u < kAttractBatch; ++u) {
        float ax = 0.0f, ay = 0.0f;
        if (has[u]) add_four(c[u], p[u], pos, ax, ay);
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
template <int STRIDE>
__device__ __forceinline__ void attract_long_row(uint32_t b, uint32_t e, int first, float2 p,
                                                 const float2 *__restrict pos,
                                                 const int4 *__restrict col4, float &ax,
                                                 float &ay) {
    uint32_t q = b + first;
    for (; q + 3 * STRIDE < e; q += 4 * STRIDE) {
        const int4 c0 = __ldcs(&col4[q]), c1 = __ldcs(&col4[q + STRIDE]);
        const int4 c2 = __ldcs(&col4[q + 2 * STRIDE]), c3 = __ldcs(&col4[q + 3 * STRIDE]);
        add_four(c0, p, pos, ax, ay);
        add_four(c1, p, pos, ax, ay);
        add_four(c2, p, pos, ax, ay);
        add_four(c3, p, pos, ax, ay);
    }
    for (; q < e; q += STRIDE) add_four(__ldcs(&col4[q]), p, pos, ax, ay);
}

__global__ void __launch_bounds__(256) k_attract(AttractPlan plan, const float2 *__restrict pos,
                                                 const float *__restrict mass,
                                                 const uint32_t *__restrict off,
                                                 const int4 *__restrict col4,
                                                 float2 *__restrict fag, Params prm) {
    __shared__ float2 s_red[256 / kWarp];
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
        const float2 p = pos[row];
        float ax = 0.0f, ay = 0.0f;
        attract_long_row<256>(off[row] >> 2, off[row + 1] >> 2, threadIdx.x, p, pos, col4, ax, ay);
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
        const float2 p = pos[row];
        float ax = 0.0f, ay = 0.0f;
        attract_long_row<32>(off[row] >> 2, off[row + 1] >> 2, lane, p, pos, col4, ax, ay);
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
        case 16: attract_short_rows<16>(row0, bk.row_end, pos, mass, off, col4, fag, prm, lane); break;
        case 8: attract_short_rows<8>(row0, bk.row_end, pos, mass, off, col4, fag, prm, lane); break;
        case 4: attract_short_rows<4>(row0, bk.row_end, pos, mass, off, col4, fag, prm, lane); break;
        case 2: attract_short_rows<2>(row0, bk.row_end, pos, mass, off, col4, fag, prm, lane); break;
        default: attract_short_rows<1>(row0, bk.row_end, pos, mass, off, col4, fag, prm, lane); break;
    }
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
    k_keys<<<sort_tiles(b.n), 256, 0, s>>>(b.n, b.pos, b.st, b.keys[0], b.vals[0], b.ctr,
                                           b.sort_counts);
}

void launch_runs(const Buffers &b, int perturb, int nsm, cudaStream_t s) {
    k_runs<<<grid_for(b.n, 256, nsm * 8), 256, 0, s>>>(b.n, b.keys[0], b.vals[0], b.pos, b.ref_of,
                                                       b.st, perturb);
}

void launch_tree_count(const Buffers &b, cudaStream_t s) {
    k_tree_count<<<count_tiles(b.n), kCountThreads, 0, s>>>(
        b.n, b.keys[0], b.lcp, b.group, b.cnt, b.kids, b.capacity, b.st, b.ctr, b.count_status,
        b.vals[0], b.pos, b.ref_of);
}

void launch_emit(const Buffers &b, int nsm, cudaStream_t s) {
    k_emit<<<grid_for(b.n, 256, nsm * 8), 256, 0, s>>>(b.n, b.keys[0], b.vals[0], b.lcp, b.group,
                                                       b.pos, b.mass, b.nodes, b.parent, b.cnt, b.kids,
                                                       b.body_node, b.st);
}

void launch_summarize(const Buffers &b, int nsm, cudaStream_t s) {
    k_summarize<<<grid_for(b.n, 256, nsm * 8), 256, 0, s>>>(b.n, b.body_node, b.parent, b.cnt, b.kids,
                                                            b.nodes, b.st);
}

void launch_traverse(const Buffers &b, const Params &p, int nblocks, cudaStream_t s) {
    k_traverse<<<nblocks, kTravThreads, 0, s>>>(b.n, b.nodes, b.body_node, b.vals[0], b.fag,
                                                b.fprev, b.f, b.warp_partial, b.st, b.ctr, p);
}

void launch_displace(const Buffers &b, int nsm, cudaStream_t s) {
    k_displace<<<grid_for(b.n, kDispThreads, nsm * 4), kDispThreads, 0, s>>>(
        b.n, b.pos, b.f, b.fprev, b.bbox_partial, b.st, b.ctr);
}

void launch_attract(const Buffers &b, const Params &p, const AttractPlan &plan, cudaStream_t s) {
    if (plan.nblocks == 0) return;
    k_attract<<<plan.nblocks, 256, 0, s>>>(plan, b.pos, b.mass, b.csr_off, b.csr_col4, b.fag, p);
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
    int nb = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_traverse, kTravThreads, 0);
    return nb < 1 ? 1 : nb;
}

}  // namespace fa2
