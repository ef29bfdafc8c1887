// fa2_device.cuh -- small device helpers shared by the kernel files.
#pragma once

#include <float.h>
#include <stdint.h>

#include "fa2_internal.cuh"

namespace fa2 {

constexpr unsigned kFullMask = 0xffffffffu;

// Common leading quadrant digits of two 32-digit Morton keys (32 if equal).
__device__ __forceinline__ int lcp_digits(uint64_t a, uint64_t b) {
    const uint64_t x = a ^ b;
    return x == 0 ? kLevels : (__clzll(x) >> 1);
}

// Tree node meta word: next index (node after the subtree) << 6 | level code.
__device__ __forceinline__ int meta_level(int meta) { return meta & 63; }
__device__ __forceinline__ uint32_t meta_next(int meta) { return (uint32_t)meta >> kMetaShift; }
__device__ __forceinline__ float make_meta(uint32_t next, int level) {
    return __int_as_float((int)((next << kMetaShift) | (uint32_t)level));
}


// Softened squared distance dx^2 + dy^2 + eps of the walk, with every
// rounding spelled out so that each kernel that restates it gets the same
// bits whatever the compiler would contract.
__device__ __forceinline__ float sq_dist(float dx, float dy, float eps) {
    return __fadd_rn(__fmaf_rn(dx, dx, __fmul_rn(dy, dy)), eps);
}

// dx^2 + dy^2 with the same spelled-out roundings (the swing and traction
// terms of the passes that end an iteration).
__device__ __forceinline__ float sq_norm(float dx, float dy) {
    return __fmaf_rn(dx, dx, __fmul_rn(dy, dy));
}

// prevent_overlap (the option src/RPForceAtlas2.hpp:44 declares and the
// reference never implements, src/RPCPUForceAtlas2.cpp:201-205): the rule of
// the ForceAtlas2 paper (Jacomy et al., PLoS ONE 2014) on the border-to-
// border distance d' = d - s_i - s_j, with d the walk's softened distance
// sqrt(d^2 + eps).  Repulsion k_r m_i m_j / d' while apart, 100 k_r m_i m_j
// while overlapping, nothing at d' = 0; returned as the factor c of
// k_r m_i c (p_i - p_j).
__device__ __forceinline__ float overlap_factor(float d2, float si, float sj, float mj) {
    const float ds = sqrtf(d2);
    const float dp = ds - si - sj;
    if (dp > 0.0f) return mj / (ds * dp);
    if (dp < 0.0f) return 100.0f * mj / ds;
    return 0.0f;
}

// --------------------------------------------------- shared by the kernels --

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


// One neighbour's pull: p_j - p_i, or with linear-log attraction (use_linlog
// of the reference's CPU path, RPCPUForceAtlas2.cpp:59-67) that vector times
// log(1 + d) / d, d = 0 taken as FLT_MAX (padding ids give the zero vector).
// The product is rounded on its own (__fmul_rn, never fused into the sum that
// follows), as the reference's CPU code rounds it before adding.
template <bool LINLOG>
__device__ __forceinline__ float2 pull(float2 q, float2 p) {
    float dx = q.x - p.x, dy = q.y - p.y;
    if (LINLOG) {
        const float ex = p.x - q.x, ey = p.y - q.y;
        const float dist = sqrtf(ex * ex + ey * ey);
        const float w = dist == 0.0f ? FLT_MAX : logf(1 + dist) / dist;
        dx = __fmul_rn(dx, w);
        dy = __fmul_rn(dy, w);
    }
    return make_float2(dx, dy);
}


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
__device__ __forceinline__ bool deep_less(float2 pa, float2 pb, uint32_t ida, uint32_t idb, float x, float y,
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
    const unsigned long long lo2 = __shfl_up_sync(kFullMask, lo, o);
    const long long hi2 = __shfl_up_sync(kFullMask, hi, o);
    return ((i128)hi2 << 64) | (i128)lo2;
}

__device__ __forceinline__ i128 shfl_xor_i128(i128 v, int o) {
    const unsigned long long lo = (unsigned long long)v;
    const long long hi = (long long)(v >> 64);
    const unsigned long long lo2 = __shfl_xor_sync(kFullMask, lo, o);
    const long long hi2 = __shfl_xor_sync(kFullMask, hi, o);
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
__device__ __forceinline__ int find_end(const uint64_t *__restrict keys, const int8_t *__restrict lcp, int n,
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


// The adaptive speed rule (SpeedKernel's last part, src/RPFA2Kernels.cu:177-219
// = RPCPUForceAtlas2.cpp:162-196) from the summed swing and traction of the n
// bodies: updates the speed efficiency se and the global speed gs.
__device__ __forceinline__ void speed_update(float swg, float etra, int n, float jitter_tolerance,
                                             float k_s_max, float &se, float &gs) {
    float estimated_optimal_jitter_tollerance = 0.05 * sqrtf((float)n);
    float minJT = sqrtf(estimated_optimal_jitter_tollerance);
    float jt = jitter_tolerance *
               fmaxf(minJT, fminf(k_s_max, estimated_optimal_jitter_tollerance * etra /
                                               powf((float)n, 2.0f)));
    float min_speed_efficiency = 0.05f;
    if (swg / etra > 2.0) {
        if (se > min_speed_efficiency) se *= 0.5;
        jt = fmaxf(jt, jitter_tolerance);
    }
    float targetSpeed = jt * se * etra / swg;
    if (swg > jt * etra) {
        if (se > min_speed_efficiency) se *= 0.7;
    } else if (gs < 1000) {
        se *= 1.3;
    }
    float max_rise = 0.5f;
    gs += fminf(targetSpeed - gs, max_rise * gs);
}

// End of a pass that wrote one (swing, traction) partial per group of 32
// sorted bodies: the last block to finish sums the partials in a fixed order
// (thread-strided, then the warp's lanes, then the block's warps) and applies
// the speed rule (src/RPFA2Kernels.cu:177-219).  Every thread of the block
// calls it; s_last and s_red are the caller's shared memory.
template <int THREADS>
__device__ __forceinline__ void speed_finish(int n, const float2 *warp_partial, unsigned *done,
                                             DevState *st, bool &s_last,
                                             float (&s_red)[2][THREADS / kWarp]) {
    const int lane = threadIdx.x & 31;
    const int nwarps = (n + 31) >> 5;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = atomicAdd(done, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    float sw = 0.0f, tr = 0.0f;
    for (int w = threadIdx.x; w < nwarps; w += THREADS) {
        float2 v = __ldcg(&warp_partial[w]);
        sw += v.x;
        tr += v.y;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        sw += __shfl_xor_sync(kFullMask, sw, o);
        tr += __shfl_xor_sync(kFullMask, tr, o);
    }
    if (lane == 0) {
        s_red[0][threadIdx.x >> 5] = sw;
        s_red[1][threadIdx.x >> 5] = tr;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        float swg = 0.0f, etra = 0.0f;
        for (int w = 0; w < THREADS / kWarp; ++w) {
            swg += s_red[0][w];
            etra += s_red[1][w];
        }
        st->swg_sum = swg;
        st->etra_sum = etra;
        float se = st->speed_efficiency, gs = st->global_speed;
        speed_update(swg, etra, n, st->jitter_tolerance, st->k_s_max, se, gs);
        st->speed_efficiency = se;
        st->global_speed = gs;
    }
}

// Displacement factor of one body (DisplacementKernel, src/RPFA2Kernels.cu:
// 223-251): speed / (1 + sqrt(speed * |f - f_prev|)), the sum in double.
__device__ __forceinline__ float displacement_factor(float2 fi, float2 fp, float global_speed) {
    const float dx = fi.x - fp.x, dy = fi.y - fp.y;
    const float swg = sqrtf(dx * dx + dy * dy);
    return global_speed / (1.0 + sqrtf(global_speed * swg));
}

// The run of equal keys that starts at sorted body k: order it, then either
// flag exactly coincident bodies (perturb == 0) or scale every body that sits
// on an earlier one (lower reference id) by .99, as the reference's insertion
// does for the later-inserted body (src/RPBHKernels.cu:271-278).
// pos is indexed by the ids in vals; ref_of maps them to reference ids (null:
// the ids are reference ids).  The root cell is (rx, ry, rr); err and poison
// receive the kErrRunTooLong bit and the coincidence count.
__device__ __forceinline__ void fix_run(int k, int n, const uint64_t *__restrict keys,
                                        uint32_t *__restrict vals, float2 *__restrict pos,
                                        const uint32_t *__restrict ref_of, float rx, float ry,
                                        float rr, int *err, int *poison, int perturb) {
    const uint64_t key = keys[k];
    int len = 2;
    while (k + len < n && keys[k + len] == key && len <= kMaxRun) ++len;
    if (len > kMaxRun) {
        atomicOr(err, kErrRunTooLong);
        return;
    }
    float cx, cy, cr;
    key_centre(key, rx, ry, rr, cx, cy, cr);
    uint32_t *v = vals + k;
    for (int a = 1; a < len; ++a) {  // insertion sort, stable
        const uint32_t va = v[a];
        const float2 pa = pos[va];
        int b = a - 1;
        while (b >= 0) {
            const uint32_t vb = v[b];
            const uint32_t ra = ref_of ? ref_of[va] : va, rb = ref_of ? ref_of[vb] : vb;
            if (!deep_less(pa, pos[vb], ra, rb, cx, cy, cr)) break;
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
    if (any && !perturb) atomicAdd(poison, 1);
}

}  // namespace fa2
