// fa2_sort.cu -- stable LSD radix sort of (64-bit Morton key, 32-bit node id)
// pairs, 8 passes of 8-bit digits, one kernel per pass.
//
// The digit histograms of all eight passes do not depend on the order of the
// keys, so k_keys (fa2_kernels.cu) counts them once while it writes the keys.
// Each pass then runs one block per 4096-key tile:
//   1. rank: every warp ranks its 512 keys by digit with __match_any_sync,
//      in key order, so equal digits keep their order (stability);
//   2. look-back: the block publishes its 256 digit counts and adds up the
//      counts of the tiles before it (decoupled look-back; tiles are numbered
//      by an atomic ticket, so every tile waited on is already running).  A
//      wait that runs past its bound sets kErrSortWait and stops the step;
//   3. scatter: keys are regrouped by digit in shared memory and written out
//      in runs, so global writes are contiguous per digit.
#include <stdint.h>

#include "fa2_internal.cuh"

namespace fa2 {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr uint32_t kFlagAgg = 1u << 30, kFlagPre = 2u << 30, kValMask = (1u << 30) - 1;

struct SortSmem {
    uint64_t keys[kSortTile];
    uint32_t vals[kSortTile];
    uint32_t whist[kSortWarps][256];  // per-warp digit counts, then offsets
    uint32_t tile_off[256];           // exclusive scan of tile digit counts
    uint32_t gbase[256];              // global start of this tile's digit run
    uint32_t scan_tmp[kSortWarps];
    int tile;
};

// Block-wide exclusive scan of one value per thread (256 threads).
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t *tmp, uint32_t *total) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(kFull, inc, o);
        if (lane >= o) inc += t;
    }
    if (lane == 31) tmp[wid] = inc;
    __syncthreads();
    uint32_t wbase = 0, all = 0;
#pragma unroll
    for (int w = 0; w < kSortWarps; ++w) {
        uint32_t t = tmp[w];
        if (w < wid) wbase += t;
        all += t;
    }
    __syncthreads();
    if (total) *total = all;
    return wbase + inc - v;
}

// Two 1024-thread blocks per SM (32 registers each) keep all tiles of a
// million-body sort resident in one wave.
__global__ void __launch_bounds__(kSortThreads, 2) k_sort_pass(
    int n, int pass, const uint64_t *__restrict kin, const uint32_t *__restrict vin,
    uint64_t *__restrict kout, uint32_t *__restrict vout, IterCounters *ctr, uint32_t *status,
    DevState *st) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SortSmem &S = *reinterpret_cast<SortSmem *>(smem_raw);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int shift = 8 * pass;
    if (st->err || st->poison) return;
    if (threadIdx.x == 0) S.tile = (int)atomicAdd(&ctr->sort_ticket[pass], 1u);
    for (int j = threadIdx.x; j < kSortWarps * 256; j += kSortThreads) (&S.whist[0][0])[j] = 0;
    __syncthreads();
    const int tile = S.tile;
    const int base = tile * kSortTile + wid * (kSortTile / kSortWarps);
    const unsigned lt_mask = (1u << lane) - 1u;

    // 1. rank within the warp's chunk, round by round
    uint64_t k[kSortRounds];
    uint32_t v[kSortRounds];
    uint32_t rank[kSortRounds];
#pragma unroll
    for (int r = 0; r < kSortRounds; ++r) {
        const int idx = base + r * 32 + lane;
        const bool valid = idx < n;
        k[r] = valid ? kin[idx] : 0ull;
        v[r] = valid ? vin[idx] : 0u;
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

    // 2. per digit (threads 0..255, thread = digit): offsets across warps,
    //    tile count, look-back
    const int d = threadIdx.x;
    const bool digit_thread = d < 256;
    uint32_t run = 0;
    if (digit_thread) {
#pragma unroll 8
        for (int w = 0; w < kSortWarps; ++w) {
            uint32_t c = S.whist[w][d];
            S.whist[w][d] = run;
            run += c;
        }
    }
    const uint32_t tile_count = run;
    uint32_t *my_status = status + (size_t)tile * 256;
    uint32_t prefix = 0;
    if (!digit_thread) {
        // no digit: only the block-wide scans below
    } else if (tile == 0) {
        atomicExch(&my_status[d], kFlagPre | tile_count);
    } else {
        atomicExch(&my_status[d], kFlagAgg | tile_count);
        int t = tile - 1;
        long spins = 0;
        while (t >= 0) {
            const uint32_t s = *((volatile uint32_t *)&status[(size_t)t * 256 + d]);
            if ((s >> 30) == 0) {
                if (++spins > (1L << 22)) {
                    atomicOr(&st->err, kErrSortWait);
                    break;
                }
                continue;
            }
            prefix += s & kValMask;
            if ((s >> 30) == 2) break;
            --t;
        }
        atomicExch(&my_status[d], kFlagPre | (prefix + tile_count));
    }
    // global start of digit d = all keys with smaller digits + earlier tiles' d
    const uint32_t hist_d = digit_thread ? ctr->hist[pass][d] : 0u;
    const uint32_t bin_base = block_excl_scan(hist_d, S.scan_tmp, nullptr);
    const uint32_t toff = block_excl_scan(tile_count, S.scan_tmp, nullptr);
    if (digit_thread) {
        S.gbase[d] = bin_base + prefix;
        S.tile_off[d] = toff;
    }
    __syncthreads();

    // 3. regroup by digit in shared memory, then write digit runs
#pragma unroll
    for (int r = 0; r < kSortRounds; ++r) {
        const int idx = base + r * 32 + lane;
        if (idx < n) {
            const uint32_t dd = (uint32_t)(k[r] >> shift) & 255u;
            const uint32_t p = S.tile_off[dd] + S.whist[wid][dd] + rank[r];
            S.keys[p] = k[r];
            S.vals[p] = v[r];
        }
    }
    __syncthreads();
    const int tile_n = min(kSortTile, n - tile * kSortTile);
    for (int j = threadIdx.x; j < tile_n; j += kSortThreads) {
        const uint64_t key = S.keys[j];
        const uint32_t dd = (uint32_t)(key >> shift) & 255u;
        const uint32_t out = S.gbase[dd] + (uint32_t)j - S.tile_off[dd];
        if (out < (uint32_t)n) {  // only false after a look-back gave up
            kout[out] = key;
            vout[out] = S.vals[j];
        }
    }
}

}  // namespace

void sort_set_smem_attr() {
    cudaFuncSetAttribute(k_sort_pass, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sizeof(SortSmem));
}

void launch_sort(const Buffers &b, cudaStream_t s) {
    const int tiles = sort_tiles(b.n);
    const size_t status_stride = (size_t)tiles * 256;
    for (int pass = 0; pass < 8; ++pass) {
        const int src = pass & 1, dst = src ^ 1;
        k_sort_pass<<<tiles, kSortThreads, sizeof(SortSmem), s>>>(
            b.n, pass, b.keys[src], b.vals[src], b.keys[dst], b.vals[dst], b.ctr,
            b.sort_status + status_stride * pass, b.st);
    }
}

}  // namespace fa2
