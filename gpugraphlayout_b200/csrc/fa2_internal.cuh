// fa2_internal.cuh -- device data layout and kernel entry points of the B200
// ForceAtlas2 engine.  Host code in fa2_capi.cu enqueues one iteration as
//
//   stream A: keys -> sort (8 passes) -> tree_count -> emit -> [join B]
//             -> traverse (+ speed) -> displace (+ next bounding box)
//   stream B: attract (gravity + attraction)
//
// which replaces the eleven launches of CUDAForceAtlas2::doStep
// (src/RPGPUForceAtlas2.cu:206-248 of the reference).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace fa2 {

constexpr int kWarp = 32;
constexpr int kLevels = 32;        // quadrant digits in a 64-bit Morton key
constexpr int kBodyLevel = 63;     // level code of a body (leaf) node
constexpr int kMetaShift = 6;      // node meta = next_index << 6 | level code
constexpr uint32_t kMaxTreeNodes = (1u << 26) - 1;  // next index fits the 26 meta bits
constexpr int kMaxRun = 1024;      // longest run of equal 64-bit keys handled
constexpr int kDeepLevels = 64;    // levels past 32 used to order such a run

// Device error bits (DevState::err).  Any of them stops the iteration.
enum : int {
    kErrScanWait = 2,      // a tree-count tile waited too long
    kErrRunTooLong = 4,    // more than kMaxRun bodies share a 64-bit key
    kErrTreeTooLarge = 8,  // the quadtree needs more nodes than allocated
    kErrNonFinite = 16,    // a position is NaN or infinite
};

// Scalars that live on the device for the whole run.
struct DevState {
    float minx, maxx, miny, maxy;        // bounding box of the positions
    float radius, rootx, rooty;          // root cell (src/RPBHKernels.cu:140-148)
    float global_speed, speed_efficiency; // src/RPFA2Kernels.cu:29-33, per context here
    float jitter_tolerance, k_s_max;
    int poison;          // coincident bodies seen: this iteration is replayed
    int err;             // kErr* bits
    int iters_done;      // completed iterations
    uint32_t tree_nodes; // nodes of the last quadtree
    int max_level;
    float swg_sum, etra_sum;
    unsigned long long interactions;  // body-node force terms of the last traversal
    unsigned long long visits;        // body-node acceptance tests of the last traversal
    float trav_radius;                // root radius the last traversal used
    int resort;                       // a sort that skipped low digits needs all of them
};

// Per-iteration scratch, cleared by one memset at the start of an iteration.
struct IterCounters {
    unsigned bbox_done;
    unsigned sort_ticket[8];
    unsigned count_ticket;
    unsigned trav_ticket;
    unsigned trav_done;
    unsigned disp_done;
    unsigned mom_ticket;
    unsigned pad[1];
    unsigned pair_count[16];  // (group, cell) pairs of a learned walk, per pair segment
    unsigned hist[8][256];  // per-pass digit histograms of the sort keys
};

// Sort geometry: one tile per block, kSortThreads threads holding `rounds`
// keys each.  The rounds (4, 5 or 6) are chosen per context so that, where
// possible, every tile gets an SM of its own (see sort_rounds).
constexpr int kSortThreads = 1024;
constexpr int kSortWarps = kSortThreads / kWarp;
constexpr int kSortMinRounds = 4;
constexpr int kSortMaxRounds = 6;
constexpr int kSortTileMin = kSortThreads * kSortMinRounds;  // 4096 keys
constexpr int kCountThreads = 256;
constexpr int kCountItems = 4;
constexpr int kCountTile = kCountThreads * kCountItems;  // 1024 bodies

inline int sort_tiles(int n, int rounds) {
    const int tile = kSortThreads * rounds;
    return (n + tile - 1) / tile;
}
// Upper bound on the tiles of any rounds choice (for sizing buffers).
inline int sort_tiles_max(int n) { return sort_tiles(n, kSortMinRounds); }
// The fewest rounds that give no more tiles than SMs; past that, the minimum.
inline int sort_rounds(int n, int nsm) {
    for (int r = kSortMinRounds; r <= kSortMaxRounds; ++r)
        if (sort_tiles(n, r) <= nsm) return r;
    return kSortMinRounds;
}
inline int count_tiles(int n) { return (n + kCountTile - 1) / kCountTile; }

// Moment scan (quadrupole option): bodies per tile and tiles.
constexpr int kMomThreads = 256;
constexpr int kMomTile = kMomThreads * 4;
inline int mom_tiles(int n) { return (n + kMomTile - 1) / kMomTile; }

// Attraction work split: rows (nodes in degree-descending order) with the
// same number of lanes per row form one contiguous bucket.
struct AttractBucket {
    int row_begin, row_end;  // rows [row_begin, row_end)
    int lanes;               // lanes per row: 256 (one block), 32, 16, ..., 1
    int block_begin;         // first block index of this bucket
};
constexpr int kMaxBuckets = 8;
constexpr int kAttractBatch = 2;  // row groups per warp in short-row buckets
struct AttractPlan {
    AttractBucket b[kMaxBuckets];
    int nbuckets;
    int nblocks;
};

// Tile sums of k_tree_count's single-pass scan (written before the tile's
// flag word is set; see fa2_tree.cu).
struct LookbackSums {
    long long agg_m, incl_m;
    __int128 agg_x, agg_y, incl_x, incl_y;
};

// Exact moments of a run of sorted bodies on the fixed-point grid of 2^-44
// root radii (q = offset from the root centre): sum m q_x, sum m q_y,
// sum m (q_x^2 - q_y^2), sum m q_x q_y.  With the total mass below 2^32 and
// |q| <= 2^45 every sum stays below 2^123.
struct Moments {
    __int128 x, y, re, im;
};

// Look-back sums of one moment tile: its own total and, once known, the
// total of every body up to its end.
struct MomLookback {
    Moments agg, incl;
};

struct Buffers {
    int n;
    // per node, internal (degree-descending) order
    float2 *pos, *fprev, *f, *fag;
    float *mass;
    const uint32_t *csr_off;  // n + 1, padded-row offsets (multiples of 4)
    const int4 *csr_col4;     // neighbour ids in fours
    const float4 *csr_w4;     // w^delta beside each id (null: unweighted, w^delta = 1)
    const uint32_t *ref_of;   // internal id -> reference id
    // sort
    uint64_t *keys[2];
    uint32_t *vals[2];
    // tree
    int8_t *lcp;              // n
    uint32_t *group;          // n: first preorder node of body k's group
    uint32_t *body_node;      // n: preorder node of sorted body k
    uint32_t *owner;          // capacity: per node, sorted body k << 6 | cell offset (63: body)
    float2 *quad;             // capacity: per cell, complex 2nd moment about its centre of mass
    Moments *pmom;            // n + 1: exclusive prefix of the body moments (quadrupole only)
    longlong2 *mom_q;         // n: sorted bodies' offsets on the 2^-44 grid (null: not kept)
    uint32_t *mom_m;          // n: sorted bodies' masses
    MomLookback *mom_lb;      // moment tiles: look-back sums
    uint32_t *mom_status;     // [moment tiles]: look-back flags (in the cleared scratch)
    float4 *nodes;            // capacity + 1: x, y, mass, meta
    uint32_t capacity;
    long long *pm;            // n + 1: exclusive prefix of mass over sorted bodies
    __int128 *pxy;            // 2(n + 1): prefix of mass x fixed-point offset, x and y
    LookbackSums *lookback;   // count tiles: tile sums of the tree-count scan
    // reductions
    float4 *bbox_partial;     // bbox blocks
    float2 *warp_partial;     // one per 32 sorted bodies
    DevState *st;
    IterCounters *ctr;
    int sort_rounds;          // keys per sort thread (tile = kSortThreads x rounds)
    int sort_first;           // first sort pass (0; 1 or 2 after shallow trees: k_fix_low)
    uint32_t *sort_counts;    // [8][sort tiles][256]: digit counts per tile and pass
    uint32_t *count_status;   // [count tiles]
    const float *size;        // n: node sizes for prevent_overlap (null: off)
    float *ssize;             // n: the same in sorted order, per iteration
};

struct Params {
    float k_r, k_g, itolsq, epssq;
    int strong_gravity;
    int linlog;     // linear-log attraction
    int multipole;  // 1: monopole cells (the reference); 2: + quadrupole term
    int nsm;
    int overlap;    // prevent_overlap: node sizes in Buffers::size
};

constexpr int kBBoxThreads = 512;
constexpr int kTravThreads = 1024;
constexpr int kDispThreads = 512;

// ---------------------------------------------------------------- kernels --
void launch_bbox(const Buffers &b, int nblocks, cudaStream_t s);
void launch_keys(const Buffers &b, int nsm, cudaStream_t s);
void launch_sort(const Buffers &b, cudaStream_t s);
void launch_fix_low(const Buffers &b, int nsm, cudaStream_t s);
// Deepest tree levels after which the next sort may skip its two lowest
// digits (levels 24..31) or its lowest one (levels 28..31): bodies then share
// at most that many digits, two levels short of the skipped ones.
constexpr int kShallowLevel = 22;
constexpr int kMidLevel = 26;
void launch_runs(const Buffers &b, int perturb, int nsm, cudaStream_t s);
void launch_tree_count(const Buffers &b, bool keep_moments, cudaStream_t s);
void launch_moments(const Buffers &b, cudaStream_t s);
void launch_emit(const Buffers &b, int nsm, cudaStream_t s);
void launch_quad_cells(const Buffers &b, int nsm, cudaStream_t s);
void launch_traverse(const Buffers &b, const Params &p, int nblocks, cudaStream_t s);
void launch_displace(const Buffers &b, int nsm, cudaStream_t s);
void launch_count_interactions(const Buffers &b, const Params &p, int nblocks, cudaStream_t s);
void launch_exact_f64(const Buffers &b, const Params &p, const uint32_t *ids, int n_ids,
                      double2 *out, cudaStream_t s);
// The accuracy guard's sums for ns samples: exact (FP64), the reference walk's
// (plain) and the applied repulsion (cur); part holds guard_part_count(ns)
// partial sums.
size_t guard_part_count(int ns);
void launch_guard(const Buffers &b, const Params &p, int ns, double2 *exact, float2 *plain,
                  float2 *cur, double2 *part, cudaStream_t s);
void launch_attract(const Buffers &b, const Params &p, const AttractPlan &plan, cudaStream_t s);
// prevent_overlap: node sizes in sorted order (before the walk)
void launch_sorted_sizes(const Buffers &b, cudaStream_t s);
void launch_scatter_xy(int n, const uint32_t *ref_of, const float2 *src_ref, float2 *dst_int,
                       cudaStream_t s);
void launch_gather_xy(int n, const uint32_t *ref_of, const float2 *src_int, float2 *dst_ref,
                      cudaStream_t s);
void launch_sorted_ref_ids(int n, const uint32_t *ref_of, const uint32_t *vals, uint32_t *out,
                           cudaStream_t s);
void sort_set_smem_attr();
int traverse_blocks_per_sm();

}  // namespace fa2
