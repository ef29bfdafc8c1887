// fa2_learn.cuh -- the learned far-field correction: data layout shared by the
// walk (fa2_kernels.cu), the MLP and training kernels (fa2_learn.cu) and the
// C ABI (fa2_capi.cu).  No counterpart in the reference, whose walk treats
// every accepted cell as a point mass (src/RPBHKernels.cu:656-668).
//
// The correction works on (group, cell) pairs: a group is the 32 sorted
// bodies one warp walks together, and the pair is a cell the whole group
// accepted that is not small for its distance (kLearnMinRatio).  For each
// pair, 12 features of the cell's multipole statistics as
// seen from the group go through a 12 -> 64 -> 64 -> 2 MLP (BF16 weights and
// activations, FP32 accumulation).  Its two outputs are the mean, over the
// group's bodies, of the error the point-mass (or quadrupole) term makes for
// that cell, in a frame turned to the cell-to-group direction and scaled by
// M / d.  Every body of the group then receives the sum of its pairs'
// corrections.
#pragma once

#include <stdint.h>

#include "fa2_internal.cuh"

namespace fa2 {

constexpr int kLearnIn = 12;      // features per pair
constexpr int kLearnInPad = 16;   // the first layer's K, padded for the MMA
constexpr int kLearnHidden = 64;  // both hidden layers
constexpr int kLearnOut = 2;
// A pair is corrected only when the group's spread (root of the mean squared
// distance of its bodies from their centroid) is at most this fraction of its
// distance to the cell: a group straddling a cell boundary sees a field that
// varies across it, which one correction per group cannot follow.
constexpr float kLearnMaxSpread = 0.5f;
// A pair is collected only when the cell's size h is at least
// kLearnMinRatio theta of its distance d from the group's centroid (feature
// 0; the walk tests the cells it accepted 32 at a time, when it writes them
// out).  The smaller cells left out carry little of the correctable error: on
// R-MAT scale 20 at theta 1.5 the pairs with h / d > 0.4 are 45 % of all and
// carry 98.6 % of the squared group-mean error, weighted as in training (0.5
// and 41 % / 98.6 % at theta 2, 0.3 and 54 % / 99.3 % at theta 1.2).
constexpr float kLearnMinRatio = 0.25f;
// Largest correction of one pair, in units of the cell's point-mass term
// M / d: the MLP's outputs (and the training targets) are clamped to it.
constexpr float kLearnMaxOut = 1.0f;

// The MLP as the kernels read it: the three weight matrices in BF16, placed
// in the tensor cores' K-major no-swizzle operand layout (8-row x 16-byte
// core matrices, the K chunks of an 8-row group 128 bytes apart, 8-row groups
// one row of chunks apart).  W1's 16 K columns are the 12 features, then the
// bias b1 split into two BF16 parts (its rounding and the rest) that meet an
// input column of ones, then zeros.  W2's 80 K columns are the 64 hidden
// units, then b2 split the same way against two more columns of ones, then
// zeros.  W3 is padded to 16 output rows (N = 16 is the smallest MMA width
// at M = 128).  b3 stays FP32.
constexpr int kLearnOutPad = 16;
constexpr int kLearnHidPad = 80;  // the second layer's K: hidden units, b2's columns
constexpr int kBiasColHi = kLearnIn, kBiasColLo = kLearnIn + 1;
constexpr int kBias2ColHi = kLearnHidden, kBias2ColLo = kLearnHidden + 1;
struct MlpDevice {
    uint16_t w1[kLearnHidden * kLearnInPad];    // 2 KB
    uint16_t w2[kLearnHidden * kLearnHidPad];   // 10 KB
    uint16_t w3[kLearnOutPad * kLearnHidden];   // 2 KB
    float b3[kLearnOut];
    float pad[2];
};

// Byte offset of element (row r, k) in a K-major no-swizzle operand tile whose
// rows hold `kchunks` 16-byte chunks of K.
__host__ __device__ constexpr uint32_t operand_offset(uint32_t r, uint32_t k, uint32_t kchunks) {
    return (r >> 3) * (kchunks * 128u) + (k >> 3) * 128u + (r & 7u) * 16u + (k & 7u) * 2u;
}

// The pair list is split into kPairSegments segments of seg_cap pairs, each
// with its own counter (IterCounters::pair_count): a warp appends to the
// segment of its warp index, so the warps' reservations spread over 16
// counters instead of queueing on one.
constexpr int kPairSegments = 16;

// What the walk of a learned iteration leaves for the MLP and the tail.
struct LearnBuffers {
    uint2 *pairs;         // (group, node) of every cell a group accepted, by segment
    uint32_t seg_cap;     // pairs per segment
    float4 *ggeo;         // 2 per group: {cx, cy, trace, lanes}, {re, im, 0, 0}
    float2 *rep;          // per sorted body: the walk's repulsion (k_r m_i applied)
    float2 *corr;         // per group: sum of its pairs' corrections (per unit k_r m_i)
    float2 *a2;           // per node: a cell's second moment as its children give it
    const MlpDevice *mlp;
};

// Device error bits of a learned iteration: more pairs than pair_cap; a wait
// for the tensor cores that gave up.
constexpr int kErrPairs = 32;
constexpr int kErrMlpWait = 64;

// ------------------------------------------------------------- launchers --

// Every cell's second moment from its children (LearnBuffers::a2), a feature
// of the pairs; after the emit, before the MLP and the training targets.
void launch_cell_a2(const Buffers &b, const LearnBuffers &lb, int nsm, cudaStream_t s);
// The MLP over every pair the walk collected: corrections summed per group.
void launch_learn_mlp(const Buffers &b, const Params &p, const LearnBuffers &lb, int nsm,
                      cudaStream_t s);
// gravity + attraction + repulsion + correction, swing/traction, speed rule.
void launch_learn_tail(const Buffers &b, const Params &p, const LearnBuffers &lb, int nsm,
                       cudaStream_t s);
// The walk of a learned iteration (k_traverse with pair collection).
void launch_traverse_learn(const Buffers &b, const Params &p, const LearnBuffers &lb,
                           int nblocks, cudaStream_t s);

// Training samples: for each pair the walk collected whose group passes the
// spread test, its 12 features, its FP64 target (the group-mean error of the
// walk's term for that cell, in the pair's frame, over M / d) and its weight
// (M/d)^2 sum of the group's squared masses, appended at *count (device).
void launch_learn_targets(const Buffers &b, const Params &p, const LearnBuffers &lb,
                          float *features, float2 *targets, float *weights, uint64_t *keys,
                          unsigned long long *count, uint64_t cap, int nsm, cudaStream_t s);

// The MLP on n rows of FP32 features (n x 12) into n x 2 outputs.
void launch_mlp_rows(const MlpDevice *mlp, const float *features, int64_t n, float2 *out,
                     int *err, int nsm, cudaStream_t s);

// One training step over `batch` samples picked by idx: forward, backward,
// weight gradients, Adam.  The parameters are FP32 (params, 5122 floats in
// the order of fa2_mlp); m and v are Adam's moments; scratch holds the
// batch's activations.
constexpr int kLearnParams = kLearnHidden * kLearnIn + kLearnHidden +
                             kLearnHidden * kLearnHidden + kLearnHidden +
                             kLearnOut * kLearnHidden + kLearnOut;
size_t learn_train_scratch_floats(int batch);
void launch_learn_train_step(float *params, float *m, float *v, int step, float lr,
                             const float *features, const float2 *targets, const float *weights,
                             float weight_scale, const uint32_t *idx, int batch, float *scratch,
                             float *loss_out, cudaStream_t s);
// Sum of n weights into *out (double).
void launch_learn_weight_sum(const float *weights, uint64_t n, double *out, cudaStream_t s);

int mlp_blocks_per_sm();
int mlp_smem_bytes_host();

}  // namespace fa2
