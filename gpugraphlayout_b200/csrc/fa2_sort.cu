// fa2_sort.cu -- stable LSD radix sort of (64-bit Morton key, 32-bit node id)
// pairs, 8 passes of 8-bit digits, one kernel per pass, no inter-block waits.
//
// The keys are cut into fixed tiles of kSortTile.  For pass p every tile
// needs, per digit, how many keys with that digit lie in the tiles before it.
// Those per-tile counts are produced one pass ahead: k_keys counts pass 0's
// digits of each tile, and the pass-p kernel, when it writes a key to its
// output position, counts the key's pass-(p+1) digit for the output tile
// (global atomics).  A tile's prefix is then a plain sum over the counts of the
// earlier tiles (read in parallel), and the global start of each digit comes
// from the all-pass histograms that k_keys also builds.  So a pass is one
// kernel with no look-back, no spin-wait and no ticket:
//   1. load the tile (all loads issued first), rank keys by digit per warp
//      with __match_any_sync in key order (stable);
//   2. per digit: offsets across warps, prefix over earlier tiles, global base;
//   3. regroup by digit in shared memory, write digit runs, count next digits.
#include <stdint.h>

#include "fa2_internal.cuh"

namespace fa2 {

namespace {

constexpr unsigned kFull = 0xffffffffu;

struct SortSmem {
    uint64_t keys[kSortTile];
    uint32_t vals[kSortTile];
    uint32_t whist[kSortWarps][256];  // per-warp digit counts, then offsets
    uint32_t tile_off[256];           // exclusive scan of tile digit counts
    uint32_t gbase[256];              // global start of this tile's digit run
    uint32_t part[kSortThreads / 256][256];  // partial prefixes over earlier tiles
    uint32_t scan_tmp[kSortWarps];
};

// Block-wide exclusive scan of one value per thread.
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t *tmp) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(kFull, inc, o);
        if (lane >= o) inc += t;
    }
    if (lane == 31) tmp[wid] = inc;
    __syncthreads();
    uint32_t wbase = 0;
    for (int w = 0; w < wid; ++w) wbase += tmp[w];
    __syncthreads();
    return wbase + inc - v;
}

__global__ void __launch_bounds__(kSortThreads, 2) k_sort_pass(
    int n, int pass, const uint64_t *__restrict kin, const uint32_t *__restrict vin,
    uint64_t *__restrict kout, uint32_t *__restrict vout, const IterCounters *__restrict ctr,
    uint32_t *__restrict counts, int ntiles, const DevState *__restrict st) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SortSmem &S = *reinterpret_cast<SortSmem *>(smem_raw);
    if (st->err || st->poison) return;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int shift = 8 * pass;
    const int tile = blockIdx.x;
    for (int j = threadIdx.x; j < kSortWarps * 256; j += kSortThreads) (&S.whist[0][0])[j] = 0;
    const int base = tile * kSortTile + wid * (kSortTile / kSortWarps);
    const unsigned lt_mask = (1u << lane) - 1u;

    // 0. this tile's prefix per digit: the counts of all earlier tiles, summed
    //    by 4 threads per digit with 8 loads in flight each, started first so
    //    that the loads overlap the ranking below
    uint32_t prefix_part;
    {
        const uint32_t *cp = counts + (size_t)pass * ntiles * 256 + (threadIdx.x & 255);
        uint32_t a[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        int t = threadIdx.x >> 8;
        for (; t + 28 < tile; t += 32) {
#pragma unroll
            for (int j = 0; j < 8; ++j) a[j] += __ldcg(cp + (size_t)(t + 4 * j) * 256);
        }
        for (; t < tile; t += 4) a[0] += __ldcg(cp + (size_t)t * 256);
        prefix_part = ((a[0] + a[1]) + (a[2] + a[3])) + ((a[4] + a[5]) + (a[6] + a[7]));
    }

    // 1. load the warp's chunk (all loads in flight), then rank round by round
    uint64_t k[kSortRounds];
    uint32_t v[kSortRounds];
#pragma unroll
    for (int r = 0; r < kSortRounds; ++r) {
        const int idx = base + r * 32 + lane;
        k[r] = idx < n ? kin[idx] : 0ull;
        v[r] = idx < n ? vin[idx] : 0u;
    }
    __syncthreads();
    uint32_t rank[kSortRounds];
#pragma unroll
    for (int r = 0; r < kSortRounds; ++r) {
        const bool valid = base + r * 32 + lane < n;
        const uint32_t d = valid ? (uint32_t)(k[r] >> shift) & 255u : 256u + lane;
        const unsigned peers = __match_any_sync(kFull, d);
        uint32_t before = 0;
        if (valid) before = S.whist[wid][d];
        rank[r] = before + __popc(peers & lt_mask);
        __syncwarp();
        if (valid && (peers & lt_mask) == 0) S.whist[wid][d] = before + __popc(peers);
        __syncwarp();
    }
    __syncthreads();

    // 2. per digit (threads 0..255): offsets across warps, prefix over the
    //    earlier tiles, global start
    const int d = threadIdx.x;
    const bool digit_thread = d < 256;
    S.part[threadIdx.x >> 8][threadIdx.x & 255] = prefix_part;
    __syncthreads();
    uint32_t tile_count = 0, prefix = 0, hist_d = 0;
    if (digit_thread) {
#pragma unroll 8
        for (int w = 0; w < kSortWarps; ++w) {
            const uint32_t c = S.whist[w][d];
            S.whist[w][d] = tile_count;
            tile_count += c;
        }
        prefix = (S.part[0][d] + S.part[1][d]) + (S.part[2][d] + S.part[3][d]);
        hist_d = ctr->hist[pass][d];
    }
    const uint32_t bin_base = block_excl_scan(hist_d, S.scan_tmp);
    const uint32_t toff = block_excl_scan(tile_count, S.scan_tmp);
    if (digit_thread) {
        S.gbase[d] = bin_base + prefix;
        S.tile_off[d] = toff;
    }
    __syncthreads();

    // 3. regroup by digit in shared memory, then write digit runs and count
    //    the next pass's digits per output tile
#pragma unroll
    for (int r = 0; r < kSortRounds; ++r) {
        if (base + r * 32 + lane < n) {
            const uint32_t dd = (uint32_t)(k[r] >> shift) & 255u;
            const uint32_t p = S.tile_off[dd] + S.whist[wid][dd] + rank[r];
            S.keys[p] = k[r];
            S.vals[p] = v[r];
        }
    }
    __syncthreads();
    const int tile_n = min(kSortTile, n - tile * kSortTile);
    uint32_t *next = pass < 7 ? counts + (size_t)(pass + 1) * ntiles * 256 : nullptr;
    for (int j = threadIdx.x; j < tile_n; j += kSortThreads) {
        const uint64_t key = S.keys[j];
        const uint32_t dd = (uint32_t)(key >> shift) & 255u;
        const uint32_t out = S.gbase[dd] + (uint32_t)j - S.tile_off[dd];
        kout[out] = key;
        vout[out] = S.vals[j];
        if (next)
            atomicAdd(&next[(size_t)(out / kSortTile) * 256 + ((uint32_t)(key >> (shift + 8)) & 255u)], 1u);
    }
}

}  // namespace

void sort_set_smem_attr() {
    cudaFuncSetAttribute(k_sort_pass, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sizeof(SortSmem));
}

void launch_sort(const Buffers &b, cudaStream_t s) {
    const int tiles = sort_tiles(b.n);
    for (int pass = 0; pass < 8; ++pass) {
        const int src = pass & 1, dst = src ^ 1;
        k_sort_pass<<<tiles, kSortThreads, sizeof(SortSmem), s>>>(
            b.n, pass, b.keys[src], b.vals[src], b.keys[dst], b.vals[dst], b.ctr, b.sort_counts,
            tiles, b.st);
    }
}

}  // namespace fa2
