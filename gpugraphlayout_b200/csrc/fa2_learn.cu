// fa2_learn.cu -- the learned far-field correction's kernels: pair features,
// the MLP on the tensor cores (tcgen05, accumulators in tensor memory), the
// FP64 training targets, the FP32 training step (forward, backward, Adam),
// and the tail of a learned iteration (forces, swing/traction, speed rule).
// No counterpart in the reference: its walk adds every accepted cell as a
// point mass (src/RPBHKernels.cu:656-668), which is the term corrected here.
#include <cuda_bf16.h>
#include <stdint.h>
#include <stdio.h>

#include <algorithm>
#include <cmath>

#include "fa2_device.cuh"
#include "fa2_learn.cuh"

namespace fa2 {

namespace {

constexpr unsigned kFull = kFullMask;

// ------------------------------------------------------------- features --

// The complex second moment of a cell about its centre of mass Z as its
// children (at most four, in preorder after the cell; the first four bodies
// of a run of coincident keys) give it: sum_c m_c (z_c - Z)^2.  It leaves out
// each child's own second moment, so it is a feature, not the quadrupole
// term; it needs no moment scan, only the tree.
__device__ __forceinline__ float2 children_a2(const float4 *__restrict nodes, uint32_t g,
                                              float4 cell) {
    const uint32_t end = meta_next(__float_as_int(cell.w));
    uint32_t c = g + 1;
    float ar = 0.0f, ai = 0.0f;
#pragma unroll 1
    for (int q = 0; q < 4 && c < end; ++q) {
        const float4 ch = nodes[c];
        const float dx = ch.x - cell.x, dy = ch.y - cell.y;
        ar = fmaf(ch.z, dx * dx - dy * dy, ar);
        ai = fmaf(ch.z, 2.0f * dx * dy, ai);
        c = meta_next(__float_as_int(ch.w));  // the node after the child's subtree
    }
    return make_float2(ar, ai);
}

// children_a2 of every cell of the tree, one thread per node; bodies are
// skipped (no pair has one).
__global__ void __launch_bounds__(256) k_cell_a2(const float4 *__restrict nodes,
                                                 const DevState *st, float2 *__restrict a2) {
    if (st->err || st->poison) return;
    const uint32_t end = st->tree_nodes;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x + 1; i < end;
         i += gridDim.x * blockDim.x) {
        const float4 cell = nodes[i];
        if (meta_level(__float_as_int(cell.w)) != kBodyLevel) a2[i] = children_a2(nodes, i, cell);
    }
}

// The 12 features of a (group, cell) pair, in the frame turned so that the
// direction from the cell's centre of mass Z to the group's centroid g is the
// first axis, lengths over d = |g - Z|:
//   0  h / d               cell width h = 2 radius / 2^level
//   1  s / d               group spread s (root of the mean squared distance
//                          of its bodies from g)
//   2,3 a2 / (M d^2)       the cell's complex second moment about Z as its
//                          children give it (children_a2), turned
//   4,5 b2 / d^2           the group's complex second moment about g, turned
//   6  |a2| / (M h^2)      how far the cell's mass sits from its centre
//   7  log2(d^2 / dq) / 8  margin over the walk's acceptance threshold dq
//   8  (h / d)^2
//   9  (s / d)^2
//   10 log2(1 + s / h) / 8
//   11 bodies in the group / 32
// Every feature is a ratio of lengths (or of moments to the matching power
// of a length), so a model trained on one graph size serves another: the
// tree level and the cell mass themselves are not features.  Every feature
// is bounded for an accepted cell (a cell's bodies lie within sqrt(2) h of
// its centre of mass, the spread test bounds s / d); s / h alone is not (a
// tiny deep cell seen from a spread-out group), hence its logarithm.
// sig = M / d scales the outputs back, (c, s) is the turn.  Returns false
// when the pair is not corrected: a group spread beyond kLearnMaxSpread of
// the distance, or a degenerate cell or distance.
__device__ __forceinline__ bool pair_features(float4 cell, float2 a2, float4 g0, float4 g1,
                                              float radius, float itolsq, float epssq,
                                              float (&f)[kLearnIn], float &sig, float &c,
                                              float &s) {
    const int lvl = meta_level(__float_as_int(cell.w));
    const float M = cell.z;
    const float h = ldexpf(2.0f * radius, -lvl);
    const float wx = g0.x - cell.x, wy = g0.y - cell.y;
    const float d2 = wx * wx + wy * wy;
    const float spread = sqrtf(fmaxf(g0.z, 0.0f));
    if (!(d2 > epssq) || !(h > 0.0f) || !(M > 0.0f) || !(spread <= kLearnMaxSpread * sqrtf(d2))) {
#pragma unroll
        for (int q = 0; q < kLearnIn; ++q) f[q] = 0.0f;
        sig = 0.0f;
        c = 1.0f;
        s = 0.0f;
        return false;
    }
    // approximate reciprocals are enough for features; training and
    // inference compute them with this same function
    const float inv_d = rsqrtf(d2);
    c = wx * inv_d;
    s = wy * inv_d;
    const float c2 = c * c - s * s, s2 = 2.0f * c * s;
    const float a2r = a2.x * c2 + a2.y * s2, a2i = a2.y * c2 - a2.x * s2;
    const float b2r = g1.x * c2 + g1.y * s2, b2i = g1.y * c2 - g1.x * s2;
    const float inv_d2 = inv_d * inv_d;
    const float inv_md2 = __fdividef(inv_d2, M);
    const float inv_h = __fdividef(1.0f, h);
    const float dq = ldexpf(4.0f * radius * radius * itolsq, -2 * (lvl - 1)) + epssq;
    f[0] = h * inv_d;
    f[1] = spread * inv_d;
    f[2] = a2r * inv_md2;
    f[3] = a2i * inv_md2;
    f[4] = b2r * inv_d2;
    f[5] = b2i * inv_d2;
    f[6] = __fdividef(sqrtf(a2.x * a2.x + a2.y * a2.y) * inv_h * inv_h, M);
    f[7] = __log2f(__fdividef(d2, dq)) * 0.125f;
    f[8] = f[0] * f[0];
    f[9] = f[1] * f[1];
    f[10] = __log2f(1.0f + spread * inv_h) * 0.125f;
    f[11] = g0.w * (1.0f / 32.0f);
    sig = M * inv_d;
    return true;
}

// ------------------------------------------------------ tcgen05 helpers --

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory operand descriptor of the 5th-generation tensor cores: start
// address, leading byte offset (between K-adjacent core matrices) and stride
// byte offset (between 8-row groups), each in 16-byte units; descriptor
// version 1 at bit 46; no swizzle, base offset 0.
__device__ __forceinline__ uint64_t operand_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator (bit 4), BF16 A and
// B (bits 7, 10), both K-major, N >> 3 at bit 17, M >> 4 at bit 24.
constexpr uint32_t instr_desc_bf16(int m, int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) |
           ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// generic-proxy writes to shared memory made visible to the tensor cores
__device__ __forceinline__ void fence_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
        : "memory");
}

__device__ __forceinline__ bool mbar_test(uint32_t mbar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(mbar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for the phase with the given parity to complete, giving up after
// about half a second.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
    for (int i = 0; i < (1 << 22); ++i) {
        if (mbar_test(mbar, parity)) return true;
        if (i > 64) __nanosleep(128);
    }
    return false;
}

// 32 consecutive 32-bit TMEM columns of this thread's lane, waited for in the
// same statement so no use of the values can move above the wait.
__device__ __forceinline__ void tmem_load32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, "
        "[%32];\n\ttcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
          "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
          "=r"(r[31])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    __nv_bfloat162 p = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t *>(&p);
}

// max(lo, 0) and max(hi, 0) rounded to BF16 and packed, in one instruction
__device__ __forceinline__ uint32_t pack_bf16_relu(float lo, float hi) {
    uint32_t r;
    asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
    return r;
}

// 16 consecutive 32-bit TMEM columns of this thread's lane (see tmem_load32).
__device__ __forceinline__ void tmem_load16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, "
        "[%16];\n\ttcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// ------------------------------------------------------------ MLP kernel --

constexpr int kMlpRows = 128;  // rows per tile: one per TMEM lane and thread
constexpr int kMlpThreads = 128;
constexpr uint32_t kMlpTmemCols = 64;  // both layers' accumulators, in turn
constexpr uint32_t kIdesc = instr_desc_bf16(kMlpRows, kLearnHidden);
constexpr uint32_t kIdescOut = instr_desc_bf16(kMlpRows, kLearnOutPad);
constexpr int kTileChunks = kLearnHidPad / 8;  // 16-byte K chunks per row of the tile

// The tile is the A operand of all three layers, one row per thread, K-major
// with kTileChunks chunks a row: the features (chunks 0-1) for layer 1, the
// first hidden layer (chunks 0-7) and two columns of ones for b2 (chunk 8,
// written once; chunk 9 zeros) for layer 2, the second hidden layer (chunks
// 0-7) for the output layer.  Each is written after the MMAs that read the
// previous one have completed.
struct MlpSmem {
    uint8_t h[kMlpRows * kLearnHidPad * 2];   // BF16 operand tile
    MlpDevice w;                              // weights (W1, W2, W3 in operand layout)
    unsigned long long mbar;
    uint32_t tmem_base;
};
static_assert(sizeof(MlpDevice) % 16 == 0, "weights are copied in 16-byte pieces");
static_assert(offsetof(MlpSmem, h) % 16 == 0 && offsetof(MlpSmem, w) % 16 == 0,
              "operand tiles start on 16-byte boundaries");
static_assert(kLearnHidPad % 16 == 0 && kBias2ColLo < kLearnHidPad && kBias2ColHi / 8 == 8 &&
                  kBias2ColLo / 8 == 8,
              "b2's columns of ones fill the start of chunk 8");

// Writes 8 packed BF16 pairs' worth (16 bytes) as K chunk `chunk` of row r.
__device__ __forceinline__ void put_packed(uint8_t *tile, int r, int chunk, int kchunks,
                                           uint4 q) {
    *reinterpret_cast<uint4 *>(tile + operand_offset(r, chunk * 8, kchunks)) = q;
}

// Writes the 8-element K chunk `chunk` of row r (BF16) into an operand tile.
__device__ __forceinline__ void put_chunk(uint8_t *tile, int r, int chunk, int kchunks,
                                          const float *v) {
    uint4 q;
    q.x = pack_bf16(v[0], v[1]);
    q.y = pack_bf16(v[2], v[3]);
    q.z = pack_bf16(v[4], v[5]);
    q.w = pack_bf16(v[6], v[7]);
    *reinterpret_cast<uint4 *>(tile + operand_offset(r, chunk * 8, kchunks)) = q;
}

// Row r of the concatenated pair segments, as an index into the pair list:
// pre[s] is the number of rows before segment s (pre[kPairSegments] all).
__device__ __forceinline__ size_t pair_index(int64_t r, const uint32_t *pre, uint32_t seg_cap) {
    int s = 0;
#pragma unroll
    for (int q = 1; q < kPairSegments; ++q) s += (r >= (int64_t)pre[q]) ? 1 : 0;
    return (size_t)s * seg_cap + (size_t)(r - (int64_t)pre[s]);
}

// The prefix of the segments' fill (each at most seg_cap), in shared memory.
__device__ __forceinline__ void pair_prefix(const IterCounters *ctr, uint32_t seg_cap,
                                            uint32_t *pre) {
    if (threadIdx.x == 0) {
        uint32_t acc = 0;
        for (int q = 0; q < kPairSegments; ++q) {
            pre[q] = acc;
            acc += min(ctr->pair_count[q], seg_cap);
        }
        pre[kPairSegments] = acc;
    }
    __syncthreads();
}

// What one row of a tile needs: a pair, its cell, the cell's second moment
// and the group's geometry (PAIRS), or the row's features.
struct RowInputs {
    uint2 pair;
    float4 cell, g0, g1;
    float2 a2;
    float x[kLearnIn];
};

template <bool PAIRS>
__device__ __forceinline__ void load_row(RowInputs &r, int64_t row, int64_t rows,
                                         const uint32_t *pre, uint32_t seg_cap,
                                         const uint2 *__restrict pairs,
                                         const float4 *__restrict nodes,
                                         const float2 *__restrict cell_a2,
                                         const float4 *__restrict ggeo,
                                         const float *__restrict features) {
    if (row >= rows) return;
    if (PAIRS) {
        r.pair = pairs[pair_index(row, pre, seg_cap)];
        r.cell = nodes[r.pair.y];
        r.a2 = cell_a2[r.pair.y];
        r.g0 = ggeo[2 * r.pair.x];
        r.g1 = ggeo[2 * r.pair.x + 1];
    } else {
#pragma unroll
        for (int q = 0; q < kLearnIn; ++q) r.x[q] = features[row * kLearnIn + q];
    }
}

// The MLP over rows of 12 features, 128 rows per tile and thread block (one
// row per thread).  Layer 1 (K = 16: the 12 features, two columns of ones
// against b1's two BF16 parts, zeros) and layer 2 (K = 80: the 64 hidden
// units, two columns of ones against b2's parts, zeros) are 128 x 64 tcgen05
// MMAs with BF16 operands from shared memory and FP32 accumulators in tensor
// memory; each thread reads its row back with tcgen05.ld, applies ReLU and
// rounds to BF16 in one instruction per pair.  The output layer is a
// 128 x 16 MMA (W3's two rows and zeros) plus b3 in FP32.
//
// PAIRS: rows are the pairs of a learned iteration; the features come from
// the tree, the group geometry and the cell moments, and each output, turned
// back and scaled by M / d, is added to its group's correction.  Otherwise
// rows are given as FP32 features and the outputs are written out.
//
// A wait for the tensor cores that does not end within about half a second
// sets *err and ends the kernel after a second bounded wait; the tensor
// memory is released on every path.
template <bool PAIRS>
__global__ void __launch_bounds__(kMlpThreads) k_learn_mlp(
    const uint2 *__restrict pairs, const IterCounters *ctr, uint32_t seg_cap,
    const float4 *__restrict nodes, const float2 *__restrict cell_a2,
    const float4 *__restrict ggeo, const DevState *st, Params prm, float2 *__restrict corr,
    const float *__restrict features,
    int64_t nrows, float2 *__restrict out, const MlpDevice *__restrict mlp, int *err) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    MlpSmem &S = *reinterpret_cast<MlpSmem *>(smem_raw);
    __shared__ uint32_t s_pre[kPairSegments + 1];
    if (PAIRS && (st->err || st->poison)) return;
    const int t = threadIdx.x, warp = t >> 5;
    if (PAIRS) pair_prefix(ctr, seg_cap, s_pre);
    {
        const int4 *src = reinterpret_cast<const int4 *>(mlp);
        int4 *dst = reinterpret_cast<int4 *>(&S.w);
        for (int i = t; i < (int)(sizeof(MlpDevice) / 16); i += kMlpThreads) dst[i] = src[i];
    }
    // this row's columns of ones against b2 (chunk 8) and the zeros after
    // them (chunk 9); the epilogues and the features never write these chunks
    put_packed(S.h, t, kBias2ColHi / 8, kTileChunks, make_uint4(0x3F803F80u, 0u, 0u, 0u));
    put_packed(S.h, t, kBias2ColHi / 8 + 1, kTileChunks, make_uint4(0u, 0u, 0u, 0u));
    const uint32_t mbar = smem_u32(&S.mbar);
    if (t == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile(
            "tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                smem_u32(&S.tmem_base)),
            "r"(kMlpTmemCols)
            : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = S.tmem_base;
    const uint64_t dh = operand_desc(smem_u32(S.h), 128, kTileChunks * 128);
    const uint64_t dw1 = operand_desc(smem_u32(S.w.w1), 128, (kLearnInPad / 8) * 128);
    const uint64_t dw2 = operand_desc(smem_u32(S.w.w2), 128, kTileChunks * 128);
    const uint64_t dw3 = operand_desc(smem_u32(S.w.w3), 128, (kLearnHidden / 8) * 128);
    // this warp's 32 TMEM lanes (warp q of the block reads lanes 32q..32q+31)
    const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16);
    const float radius = PAIRS ? st->trav_radius : 0.0f;
    const int64_t rows = PAIRS ? (int64_t)s_pre[kPairSegments] : nrows;
    const int lane = t & 31;
    uint32_t phase = 0;
    bool bad = false;  // a wait gave up (the same for every thread)
    // The inputs of this thread's row of the next tile are loaded while the
    // tensor cores work on the current one.
    RowInputs next;
    int64_t base = (int64_t)blockIdx.x * kMlpRows;
    if (base < rows) load_row<PAIRS>(next, base + t, rows, s_pre, seg_cap, pairs, nodes, cell_a2, ggeo,
                                     features);
    for (; base < rows; base += (int64_t)gridDim.x * kMlpRows) {
        const int64_t row = base + t;
        const RowInputs in = next;
        float f[kLearnInPad];
        float sig = 0.0f, c = 1.0f, s = 0.0f;
        bool use = false;
#pragma unroll
        for (int q = kLearnIn; q < kLearnInPad; ++q) f[q] = 0.0f;
        {
            float fv[kLearnIn];
            if (row < rows) {
                if (PAIRS) {
                    use = pair_features(in.cell, in.a2, in.g0, in.g1, radius, prm.itolsq,
                                        prm.epssq, fv, sig, c, s);
                } else {
#pragma unroll
                    for (int q = 0; q < kLearnIn; ++q) fv[q] = in.x[q];
                    use = true;
                }
            } else {
#pragma unroll
                for (int q = 0; q < kLearnIn; ++q) fv[q] = 0.0f;
            }
#pragma unroll
            for (int q = 0; q < kLearnIn; ++q) f[q] = fv[q];
        }
        // the columns that meet b1's two parts in W1
        f[kBiasColHi] = 1.0f;
        f[kBiasColLo] = 1.0f;
        put_chunk(S.h, t, 0, kTileChunks, f);
        put_chunk(S.h, t, 1, kTileChunks, f + 8);
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        if (t == 0) {
            tc_fence_after();
            mma_bf16(tmem, dh, dw1, kIdesc, 0);
            mma_commit(mbar);
        }
        {
            const int64_t nb = base + (int64_t)gridDim.x * kMlpRows;
            if (nb < rows) load_row<PAIRS>(next, nb + t, rows, s_pre, seg_cap, pairs, nodes, cell_a2, ggeo,
                                        features);
        }
        // one thread waits for the tensor cores; the others wait at the
        // barrier and take no issue slots from the blocks beside them
        bool ok = t == 0 ? mbar_wait(mbar, phase) : true;
        phase ^= 1u;
        if (__syncthreads_or(!ok)) {
            bad = true;
            break;
        }
        tc_fence_after();
        // layer 1 (its bias came with the MMA): ReLU and BF16 into the
        // operand tile
#pragma unroll
        for (int half = 0; half < 2; ++half) {
            float v[32];
            tmem_load32(taddr + half * 32, v);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const float *u = v + 8 * q;
                put_packed(S.h, t, half * 4 + q, kTileChunks,
                           make_uint4(pack_bf16_relu(u[0], u[1]), pack_bf16_relu(u[2], u[3]),
                                      pack_bf16_relu(u[4], u[5]), pack_bf16_relu(u[6], u[7])));
            }
        }
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        if (t == 0) {
            tc_fence_after();
            // K = 80 in five steps of 16: the next two K chunks, 256 bytes on
#pragma unroll
            for (int kk = 0; kk < kLearnHidPad / 16; ++kk)
                mma_bf16(tmem, dh + (uint64_t)(kk * 16), dw2 + (uint64_t)(kk * 16), kIdesc,
                         kk > 0 ? 1u : 0u);
            mma_commit(mbar);
        }
        ok = t == 0 ? mbar_wait(mbar, phase) : true;
        phase ^= 1u;
        if (__syncthreads_or(!ok)) {
            bad = true;
            break;
        }
        tc_fence_after();
        // layer 2 (its bias came with the MMA): ReLU and BF16 into the
        // operand tile again (layer 2's MMAs have read it); then the output
        // layer, N = 16 of which the first two columns are W3's rows
#pragma unroll
        for (int half = 0; half < 2; ++half) {
            float v[32];
            tmem_load32(taddr + half * 32, v);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const float *u = v + 8 * q;
                put_packed(S.h, t, half * 4 + q, kTileChunks,
                           make_uint4(pack_bf16_relu(u[0], u[1]), pack_bf16_relu(u[2], u[3]),
                                      pack_bf16_relu(u[4], u[5]), pack_bf16_relu(u[6], u[7])));
            }
        }
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        if (t == 0) {
            tc_fence_after();
#pragma unroll
            for (int kk = 0; kk < kLearnHidden / 16; ++kk)
                mma_bf16(tmem, dh + (uint64_t)(kk * 16), dw3 + (uint64_t)(kk * 16), kIdescOut,
                         kk > 0 ? 1u : 0u);
            mma_commit(mbar);
        }
        ok = t == 0 ? mbar_wait(mbar, phase) : true;
        phase ^= 1u;
        if (__syncthreads_or(!ok)) {
            bad = true;
            break;
        }
        tc_fence_after();
        float y0, y1;
        {
            float v[16];
            tmem_load16(taddr, v);
            y0 = v[0] + S.w.b3[0];
            y1 = v[1] + S.w.b3[1];
        }
        if (PAIRS) {
            // a cell's correction never exceeds its own point-mass term
            // (|y| <= 1 in units of M / d); a non-finite output adds nothing
            y0 = isfinite(y0) ? fminf(fmaxf(y0, -kLearnMaxOut), kLearnMaxOut) : 0.0f;
            y1 = isfinite(y1) ? fminf(fmaxf(y1, -kLearnMaxOut), kLearnMaxOut) : 0.0f;
        }
        // the next tile's first MMA overwrites the columns just read
        tc_fence_before();
        if (PAIRS) {
            // Rows of one group are adjacent (the walk writes a group's cells
            // in runs): sum each run within the warp, one atomic per run.
            const uint32_t grp = row < rows ? in.pair.x : 0xFFFFFFFFu;
            float cx = use ? sig * (c * y0 - s * y1) : 0.0f;
            float cy = use ? sig * (s * y0 + c * y1) : 0.0f;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const float ox = __shfl_down_sync(kFull, cx, o);
                const float oy = __shfl_down_sync(kFull, cy, o);
                const uint32_t og = __shfl_down_sync(kFull, grp, o);
                if (lane + o < 32 && og == grp) {
                    cx += ox;
                    cy += oy;
                }
            }
            const uint32_t prev = __shfl_up_sync(kFull, grp, 1);
            if (grp != 0xFFFFFFFFu && (lane == 0 || prev != grp)) {
                atomicAdd(&corr[grp].x, cx);
                atomicAdd(&corr[grp].y, cy);
            }
        } else if (row < rows) {
            out[row] = make_float2(y0, y1);
        }
    }
    if (bad && t == 0) {
        atomicOr(err, kErrMlpWait);
        mbar_wait(mbar, phase ^ 1u);  // the MMAs in flight, bounded again
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(kMlpTmemCols)
                     : "memory");
    }
}

// ---------------------------------------------------------- FP64 targets --

// One warp per pair the walk collected: the group's 32 bodies (one per lane)
// against every body of the cell, whose bodies are the sorted run from the
// cell's owner to the body at the last node of its subtree.  The exact sum
// is in FP64; the walk's own term for the cell (point mass, plus the
// quadrupole term with QUAD) is restated in FP32 as the walk computes it.
// The target is the group mean of exact - term, turned into the pair's frame
// and divided by sig = M / d; the weight is sig^2 times the sum of the
// group's squared masses, the scale of the pair's share of the squared force
// error.  Samples land at *count (atomic), each with its key
// (group << 32 | node) so the host can put a snapshot's samples in a fixed
// order.
template <bool QUAD>
__global__ void __launch_bounds__(256) k_learn_targets(
    int n, const uint2 *__restrict pairs, const IterCounters *ctr, uint32_t seg_cap,
    const float4 *__restrict nodes, const float2 *__restrict quad,
    const float2 *__restrict cell_a2, const uint32_t *__restrict owner,
    const uint32_t *__restrict body_node,
    const float4 *__restrict ggeo, const DevState *st, Params prm, float *__restrict features,
    float2 *__restrict targets, float *__restrict weights, uint64_t *__restrict keys,
    unsigned long long *count, uint64_t cap) {
    __shared__ uint32_t s_pre[kPairSegments + 1];
    if (st->err || st->poison) return;
    pair_prefix(ctr, seg_cap, s_pre);
    const int lane = threadIdx.x & 31;
    const int64_t rows = (int64_t)s_pre[kPairSegments];
    const int64_t nw = (int64_t)gridDim.x * (blockDim.x >> 5);
    const float radius = st->trav_radius;
    const double eps = (double)prm.epssq;
    for (int64_t p = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; p < rows; p += nw) {
        const uint2 pr = pairs[pair_index(p, s_pre, seg_cap)];
        const uint32_t w = pr.x, node = pr.y;
        const float4 cell = nodes[node];
        const float2 a2 = cell_a2[node];
        float f[kLearnIn], sig, c, s;
        if (!pair_features(cell, a2, ggeo[2 * w], ggeo[2 * w + 1], radius, prm.itolsq,
                           prm.epssq, f, sig, c, s))
            continue;
        const uint32_t k0 = owner[node] >> 6;
        const uint32_t k1 = owner[meta_next(__float_as_int(cell.w)) - 1] >> 6;
        const int k = (int)w * 32 + lane;
        const bool active = k < n;
        const float4 me = nodes[body_node[active ? k : n - 1]];
        const double px = me.x, py = me.y;
        double ax = 0.0, ay = 0.0;
        for (uint32_t j0 = k0; j0 <= k1; j0 += 32) {
            const uint32_t jl = j0 + lane;
            const float4 o = nodes[body_node[jl <= k1 ? jl : k1]];
            const int cnt = (int)min(32u, k1 - j0 + 1);
            for (int q = 0; q < cnt; ++q) {
                const float ox = __shfl_sync(kFull, o.x, q), oy = __shfl_sync(kFull, o.y, q);
                const float om = __shfl_sync(kFull, o.z, q);
                if ((int)(j0 + q) == k) continue;
                const double dx = px - ox, dy = py - oy;
                const double cf = (double)om / (dx * dx + dy * dy + eps);
                ax += dx * cf;
                ay += dy * cf;
            }
        }
        // the walk's term for this cell (fa2_kernels.cu, k_traverse)
        const float dxf = me.x - cell.x, dyf = me.y - cell.y;
        const float d2f = sq_dist(dxf, dyf, prm.epssq);
        float bx, by;
        if (QUAD) {
            const float inv = __fdividef(1.0f, d2f);
            const float cm = cell.z * inv;
            bx = dxf * cm;
            by = dyf * cm;
            const float ux = dxf * inv, uy = dyf * inv;
            const float xx = ux * ux, yy = uy * uy;
            const float ur = ux * fmaf(-3.0f, yy, xx);
            const float ui = uy * fmaf(-3.0f, xx, yy);
            const float2 q = quad[node];  // the walk's own (exact) a2
            bx = fmaf(q.x, ur, fmaf(-q.y, ui, bx));
            by = fmaf(-q.x, ui, fmaf(-q.y, ur, by));
        } else {
            const float cm = __fdividef(cell.z, d2f);
            bx = dxf * cm;
            by = dyf * cm;
        }
        double rx = active ? ax - (double)bx : 0.0, ry = active ? ay - (double)by : 0.0;
        double m2 = active ? (double)me.z * me.z : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            rx += __shfl_xor_sync(kFull, rx, o);
            ry += __shfl_xor_sync(kFull, ry, o);
            m2 += __shfl_xor_sync(kFull, m2, o);
        }
        if (lane == 0) {
            const double lanes = (double)min(32, n - (int)w * 32);
            const double mx = rx / lanes, my = ry / lanes;
            const unsigned long long idx = atomicAdd(count, 1ull);
            if (idx < cap) {
#pragma unroll
                for (int q = 0; q < kLearnIn; ++q) features[idx * kLearnIn + q] = f[q];
                // within the bound the MLP's outputs are held to
                const double lim = (double)kLearnMaxOut;
                targets[idx] = make_float2((float)fmin(fmax((c * mx + s * my) / sig, -lim), lim),
                                           (float)fmin(fmax((c * my - s * mx) / sig, -lim), lim));
                weights[idx] = (float)((double)sig * sig * m2);
                keys[idx] = (uint64_t)w << 32 | node;
            }
        }
    }
}

// --------------------------------------------------------------- training --

// Parameter offsets in the FP32 parameter vector (the order of fa2_mlp).
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kLearnHidden * kLearnIn;
constexpr int kOffW2 = kOffB1 + kLearnHidden;
constexpr int kOffB2 = kOffW2 + kLearnHidden * kLearnHidden;
constexpr int kOffW3 = kOffB2 + kLearnHidden;
constexpr int kOffB3 = kOffW3 + kLearnOut * kLearnHidden;
static_assert(kOffB3 + kLearnOut == kLearnParams, "parameter layout");
// Largest weight a sample gets once scaled to a unit mean.
constexpr float kMaxSampleWeight = 100.0f;
// Per-sample activations kept for the weight gradients.
constexpr int kActX = 0, kActH1 = kLearnIn, kActH2 = kActH1 + kLearnHidden,
              kActDY = kActH2 + kLearnHidden, kActDH2 = kActDY + kLearnOut,
              kActDH1 = kActDH2 + kLearnHidden, kActStride = kActDH1 + kLearnHidden;
constexpr int kTrainThreads = 128;

// Forward and backward pass of one sample per thread, FP32 throughout.  The
// loss is sum_s w_s |y_s - t_s|^2 / (2 batch) (the mean over the batch's
// output elements, weighted); the activations, the output gradient and the
// hidden-layer gradients go to the sample's row of act.
__global__ void __launch_bounds__(kTrainThreads) k_train_fwd(
    const float *__restrict params, const float *__restrict features,
    const float2 *__restrict targets, const float *__restrict weights, float wscale,
    const uint32_t *__restrict idx, int batch, float *__restrict act,
    float *__restrict loss_part) {
    __shared__ float P[kLearnParams];
    __shared__ float s_loss[kTrainThreads / kWarp];
    for (int i = threadIdx.x; i < kLearnParams; i += kTrainThreads) P[i] = params[i];
    __syncthreads();
    const int b = blockIdx.x * kTrainThreads + threadIdx.x;
    float l = 0.0f;
    if (b < batch) {
        const uint32_t sidx = idx ? idx[b] : (uint32_t)b;
        float *row = act + (size_t)b * kActStride;
        float x[kLearnIn];
#pragma unroll
        for (int q = 0; q < kLearnIn; ++q) x[q] = features[(size_t)sidx * kLearnIn + q];
        const float2 t = targets[sidx];
        const float w = fminf(weights[sidx] * wscale, kMaxSampleWeight);
        // h1 in registers; h2 one unit at a time into the sample's row (read
        // back for the backward pass), so no more than two 64-vectors are live
        float h1[kLearnHidden];
#pragma unroll
        for (int j = 0; j < kLearnHidden; ++j) {
            float a = P[kOffB1 + j];
#pragma unroll
            for (int q = 0; q < kLearnIn; ++q) a = fmaf(P[kOffW1 + j * kLearnIn + q], x[q], a);
            h1[j] = fmaxf(a, 0.0f);
        }
#pragma unroll
        for (int q = 0; q < kLearnIn; ++q) row[kActX + q] = x[q];
#pragma unroll
        for (int q = 0; q < kLearnHidden; ++q) row[kActH1 + q] = h1[q];
        float y0 = P[kOffB3], y1 = P[kOffB3 + 1];
#pragma unroll 1
        for (int j = 0; j < kLearnHidden; ++j) {
            float a = P[kOffB2 + j];
#pragma unroll
            for (int q = 0; q < kLearnHidden; ++q)
                a = fmaf(P[kOffW2 + j * kLearnHidden + q], h1[q], a);
            const float h2 = fmaxf(a, 0.0f);
            row[kActH2 + j] = h2;
            y0 = fmaf(P[kOffW3 + j], h2, y0);
            y1 = fmaf(P[kOffW3 + kLearnHidden + j], h2, y1);
        }
        const float e0 = y0 - t.x, e1 = y1 - t.y;
        l = w * (e0 * e0 + e1 * e1);
        const float dy0 = w * e0 / (float)batch, dy1 = w * e1 / (float)batch;
        row[kActDY] = dy0;
        row[kActDY + 1] = dy1;
        // dh2 unit by unit, accumulated into dh1 = W2^T dh2 over the units
        float g1[kLearnHidden];
#pragma unroll
        for (int q = 0; q < kLearnHidden; ++q) g1[q] = 0.0f;
#pragma unroll 1
        for (int j = 0; j < kLearnHidden; ++j) {
            const float dh2 = row[kActH2 + j] > 0.0f
                                  ? fmaf(P[kOffW3 + j], dy0, P[kOffW3 + kLearnHidden + j] * dy1)
                                  : 0.0f;
            row[kActDH2 + j] = dh2;
#pragma unroll
            for (int q = 0; q < kLearnHidden; ++q)
                g1[q] = fmaf(P[kOffW2 + j * kLearnHidden + q], dh2, g1[q]);
        }
#pragma unroll
        for (int q = 0; q < kLearnHidden; ++q) row[kActDH1 + q] = h1[q] > 0.0f ? g1[q] : 0.0f;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(kFull, l, o);
    if ((threadIdx.x & 31) == 0) s_loss[threadIdx.x >> 5] = l;
    __syncthreads();
    if (threadIdx.x == 0) {
        float sum = 0.0f;
        for (int q = 0; q < kTrainThreads / kWarp; ++q) sum += s_loss[q];
        loss_part[blockIdx.x] = sum / (2.0f * (float)batch);
    }
}

// Gradient of every parameter over the batch (fixed summation order) and
// Adam's update (PyTorch's form: m and v moments, bias corrections bc1 and
// sqrt(bc2), eps added to sqrt(v) / sqrt(bc2)).  One block per output unit of
// a layer; thread j < inputs handles W[unit][j], thread `inputs` the bias.
constexpr int kGradThreads = 96;
__global__ void __launch_bounds__(kGradThreads) k_train_grad_adam(
    float *__restrict params, float *__restrict m, float *__restrict v, const float *__restrict act,
    int batch, float lr, float bc1, float bc2_sqrt, const float *__restrict loss_part,
    int loss_blocks, float *loss_out) {
    int unit = blockIdx.x, nin, in_off, d_off, p_w, p_b;
    if (unit < kLearnHidden) {
        nin = kLearnIn;
        in_off = kActX;
        d_off = kActDH1 + unit;
        p_w = kOffW1 + unit * kLearnIn;
        p_b = kOffB1 + unit;
    } else if (unit < 2 * kLearnHidden) {
        unit -= kLearnHidden;
        nin = kLearnHidden;
        in_off = kActH1;
        d_off = kActDH2 + unit;
        p_w = kOffW2 + unit * kLearnHidden;
        p_b = kOffB2 + unit;
    } else {
        unit -= 2 * kLearnHidden;
        nin = kLearnHidden;
        in_off = kActH2;
        d_off = kActDY + unit;
        p_w = kOffW3 + unit * kLearnHidden;
        p_b = kOffB3 + unit;
    }
    const int j = threadIdx.x;
    if (j <= nin) {
        float g0 = 0.0f, g1 = 0.0f, g2 = 0.0f, g3 = 0.0f;
        int b = 0;
        for (; b + 4 <= batch; b += 4) {
            const float *r = act + (size_t)b * kActStride;
            const float i0 = j < nin ? r[in_off + j] : 1.0f;
            const float i1 = j < nin ? r[kActStride + in_off + j] : 1.0f;
            const float i2 = j < nin ? r[2 * kActStride + in_off + j] : 1.0f;
            const float i3 = j < nin ? r[3 * kActStride + in_off + j] : 1.0f;
            g0 = fmaf(r[d_off], i0, g0);
            g1 = fmaf(r[kActStride + d_off], i1, g1);
            g2 = fmaf(r[2 * kActStride + d_off], i2, g2);
            g3 = fmaf(r[3 * kActStride + d_off], i3, g3);
        }
        for (; b < batch; ++b) {
            const float *r = act + (size_t)b * kActStride;
            g0 = fmaf(r[d_off], j < nin ? r[in_off + j] : 1.0f, g0);
        }
        const float g = (g0 + g1) + (g2 + g3);
        const int p = j < nin ? p_w + j : p_b;
        const float mv = 0.9f * m[p] + (1.0f - 0.9f) * g;
        const float vv = 0.999f * v[p] + (1.0f - 0.999f) * g * g;
        m[p] = mv;
        v[p] = vv;
        const float denom = sqrtf(vv) / bc2_sqrt + 1e-8f;
        params[p] -= (lr / bc1) * (mv / denom);
    }
    if (loss_out && blockIdx.x == 0 && threadIdx.x == 0) {
        float sum = 0.0f;
        for (int q = 0; q < loss_blocks; ++q) sum += loss_part[q];
        *loss_out = sum;
    }
}

__global__ void k_weight_sum(const float *__restrict w, uint64_t n, double *out) {
    __shared__ double s[1024 / kWarp];
    double a = 0.0;
    for (uint64_t i = threadIdx.x; i < n; i += blockDim.x) a += (double)w[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(kFull, a, o);
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = a;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) t += s[q];
        *out = t;
    }
}

// ------------------------------------------------------------------ tail --

// The end of a learned iteration, one warp per group of 32 sorted bodies:
// the total force (gravity + attraction, the walk's repulsion, and k_r m_i
// times the group's correction), swing and traction per warp and, in the
// last block, the speed rule -- the tail of k_traverse, so an all-zero
// correction gives the plain iteration's forces and speed bit for bit.
__global__ void __launch_bounds__(kTravThreads, 2048 / kTravThreads) k_learn_tail(
    int n, const float4 *__restrict nodes, const uint32_t *__restrict body_node,
    const uint32_t *__restrict vals, const float2 *__restrict fag,
    const float2 *__restrict fprev, float2 *__restrict f, float2 *__restrict warp_partial,
    const float2 *__restrict rep, const float2 *__restrict corr, DevState *st,
    IterCounters *ctr, Params prm) {
    __shared__ bool s_last;
    __shared__ float s_red[2][kTravThreads / kWarp];
    if (st->err || st->poison) return;
    const int lane = threadIdx.x & 31;
    const int nwarps = (n + 31) >> 5;
    const int stride = (int)(gridDim.x * blockDim.x) >> 5;
    for (int w = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); w < nwarps; w += stride) {
        const int k = w * 32 + lane;
        float sw = 0.0f, tr = 0.0f;
        if (k < n) {
            const float mi = nodes[body_node[k]].z;
            const float kmi = prm.k_r * mi;
            const float2 r = rep[k], cg = corr[w];
            const uint32_t i = vals[k];
            const float2 g = fag[i], fp = fprev[i];
            float fx = g.x + r.x, fy = g.y + r.y;
            fx = fmaf(kmi, cg.x, fx);
            fy = fmaf(kmi, cg.y, fy);
            f[i] = make_float2(fx, fy);
            float dx = fx - fp.x, dy = fy - fp.y;
            sw = mi * sqrtf(sq_norm(dx, dy));
            dx = fx + fp.x;
            dy = fy + fp.y;
            tr = mi * (float)(sqrtf(sq_norm(dx, dy)) / 2.0);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            sw += __shfl_xor_sync(kFull, sw, o);
            tr += __shfl_xor_sync(kFull, tr, o);
        }
        if (lane == 0) warp_partial[w] = make_float2(sw, tr);
    }
    speed_finish<kTravThreads>(n, warp_partial, &ctr->trav_done, st, s_last, s_red);
}

// ------------------------------------------------------------- launchers --

int mlp_smem_bytes() { return (int)sizeof(MlpSmem); }

}  // namespace

int mlp_smem_bytes_host() { return mlp_smem_bytes(); }

// Blocks per SM of the MLP kernel, from its registers and shared memory and
// the SM's 512 tensor-memory columns (64 per block).  The runtime's occupancy
// query answers 1 for this kernel (it allocates tensor memory), so the limits
// are taken from the kernel's attributes and the device's properties.
int mlp_blocks_per_sm() {
    static int cached = 0;
    if (cached) return cached;
    const int bytes = mlp_smem_bytes();
    int dev = 0;
    cudaFuncAttributes fa;
    cudaDeviceProp dp;
    if (cudaFuncSetAttribute(k_learn_mlp<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             bytes) != cudaSuccess ||
        cudaFuncSetAttribute(k_learn_mlp<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             bytes) != cudaSuccess ||
        cudaGetDevice(&dev) != cudaSuccess || cudaGetDeviceProperties(&dp, dev) != cudaSuccess ||
        cudaFuncGetAttributes(&fa, k_learn_mlp<true>) != cudaSuccess) {
        const cudaError_t e = cudaGetLastError();
        fprintf(stderr, "fa2: MLP launch shape query failed (%s); 1 block per SM\n",
                cudaGetErrorString(e));
        return 1;  // not kept: the next call asks again
    }
    // per block: its shared memory plus the 1 KB the system reserves
    const size_t per_block = (size_t)bytes + fa.sharedSizeBytes + dp.reservedSharedMemPerBlock;
    int nb = (int)(dp.sharedMemPerMultiprocessor / per_block);
    const int regs = fa.numRegs * kMlpThreads;
    if (regs > 0) nb = std::min(nb, dp.regsPerMultiprocessor / regs);
    nb = std::min(nb, dp.maxThreadsPerMultiProcessor / kMlpThreads);
    nb = std::min(nb, (int)(512 / kMlpTmemCols));
    cached = std::max(nb, 1);
    return cached;
}

void launch_learn_mlp(const Buffers &b, const Params &p, const LearnBuffers &lb, int nsm,
                      cudaStream_t s) {
    k_learn_mlp<true><<<nsm * mlp_blocks_per_sm(), kMlpThreads, mlp_smem_bytes(), s>>>(
        lb.pairs, b.ctr, lb.seg_cap, b.nodes, lb.a2, lb.ggeo, b.st, p, lb.corr, nullptr, 0,
        nullptr, lb.mlp, &b.st->err);
}

void launch_mlp_rows(const MlpDevice *mlp, const float *features, int64_t n, float2 *out,
                     int *err, int nsm, cudaStream_t s) {
    if (n <= 0) return;
    const int64_t tiles = (n + kMlpRows - 1) / kMlpRows;
    const int64_t cap = (int64_t)nsm * mlp_blocks_per_sm();
    const int grid = (int)(tiles < cap ? tiles : cap);
    Params p{};
    k_learn_mlp<false><<<grid, kMlpThreads, mlp_smem_bytes(), s>>>(
        nullptr, nullptr, 0, nullptr, nullptr, nullptr, nullptr, p, nullptr, features, n, out,
        mlp, err);
}

void launch_cell_a2(const Buffers &b, const LearnBuffers &lb, int nsm, cudaStream_t s) {
    k_cell_a2<<<nsm * 8, 256, 0, s>>>(b.nodes, b.st, lb.a2);
}

void launch_learn_tail(const Buffers &b, const Params &p, const LearnBuffers &lb, int nsm,
                       cudaStream_t s) {
    k_learn_tail<<<nsm * (2048 / kTravThreads), kTravThreads, 0, s>>>(
        b.n, b.nodes, b.body_node, b.vals[0], b.fag, b.fprev, b.f, b.warp_partial, lb.rep,
        lb.corr, b.st, b.ctr, p);
}

void launch_learn_targets(const Buffers &b, const Params &p, const LearnBuffers &lb,
                          float *features, float2 *targets, float *weights, uint64_t *keys,
                          unsigned long long *count, uint64_t cap, int nsm, cudaStream_t s) {
    if (p.multipole >= 2)
        k_learn_targets<true><<<nsm * 8, 256, 0, s>>>(
            b.n, lb.pairs, b.ctr, lb.seg_cap, b.nodes, b.quad, lb.a2, b.owner, b.body_node,
            lb.ggeo,
            b.st, p, features, targets, weights, keys, count, cap);
    else
        k_learn_targets<false><<<nsm * 8, 256, 0, s>>>(
            b.n, lb.pairs, b.ctr, lb.seg_cap, b.nodes, b.quad, lb.a2, b.owner, b.body_node,
            lb.ggeo,
            b.st, p, features, targets, weights, keys, count, cap);
}

size_t learn_train_scratch_floats(int batch) {
    return (size_t)batch * kActStride + (size_t)(batch + kTrainThreads - 1) / kTrainThreads;
}

void launch_learn_train_step(float *params, float *m, float *v, int step, float lr,
                             const float *features, const float2 *targets, const float *weights,
                             float weight_scale, const uint32_t *idx, int batch, float *scratch,
                             float *loss_out, cudaStream_t s) {
    const int blocks = (batch + kTrainThreads - 1) / kTrainThreads;
    float *act = scratch;
    float *loss_part = scratch + (size_t)batch * kActStride;
    k_train_fwd<<<blocks, kTrainThreads, 0, s>>>(params, features, targets, weights,
                                                 weight_scale, idx, batch, act, loss_part);
    const double bc1 = 1.0 - std::pow(0.9, (double)step);
    const double bc2 = 1.0 - std::pow(0.999, (double)step);
    k_train_grad_adam<<<2 * kLearnHidden + kLearnOut, kGradThreads, 0, s>>>(
        params, m, v, act, batch, lr, (float)bc1, (float)std::sqrt(bc2), loss_part, blocks,
        loss_out);
}

void launch_learn_weight_sum(const float *weights, uint64_t n, double *out, cudaStream_t s) {
    k_weight_sum<<<1, 1024, 0, s>>>(weights, n, out);
}

}  // namespace fa2
