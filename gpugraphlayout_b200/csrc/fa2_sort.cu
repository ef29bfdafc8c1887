// fa2_sort.cu -- stable LSD radix sort of (64-bit Morton key, 32-bit node id)
// pairs, 8 passes of 8-bit digits, one kernel per pass, no inter-block waits.
// After a shallow tree the sort starts at pass 2 and k_fix_low orders the
// runs of keys equal in the top 48 bits (see there).
//
// The keys are cut into fixed tiles of kSortThreads x R keys (R = 4..6 rounds
// per thread, chosen per context so that the tiles fit one per SM where they
// can: a pass is one wave, and no SM runs two tiles while others idle).  For
// pass p every tile needs, per digit, how many keys with that digit lie in
// the tiles before it.  Those per-tile counts are produced one pass ahead:
// k_keys counts pass 0's digits of each tile, and the pass-p kernel, when it
// writes a key to its output position, counts the key's pass-(p+1) digit for
// the output tile (global atomics).  A tile's prefix is then a plain sum over
// the counts of the earlier tiles (read in parallel), and the global start of
// each digit comes from the all-pass histograms that k_keys also builds.  So
// a pass is one kernel with no look-back, no spin-wait and no ticket:
//   1. issue the tile's loads, then the loads of the earlier tiles' counts;
//   2. rank keys by digit per warp in key order (stable): the lanes that share
//      a digit are the AND of eight ballots, one per digit bit;
//   3. per digit: offsets across warps, prefix over earlier tiles, global base;
//   4. regroup by digit in shared memory, write digit runs, count next digits.
#include <stdint.h>

#include "fa2_internal.cuh"

namespace fa2 {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kQuarters = kSortThreads / 256;  // threads per digit in the scans

template <int R>
struct SortSmem {
    uint64_t keys[kSortThreads * R];
    uint32_t vals[kSortThreads * R];
    uint32_t whist[kSortWarps][256];    // per-warp digit counts, then offsets
    uint32_t tile_off[256];             // exclusive scan of tile digit counts
    uint32_t gbase[256];                // global start of this tile's digit run
    uint32_t part[kQuarters][256];      // partial prefixes over earlier tiles
    uint32_t qsum[kQuarters][256];      // per-quarter sums of the warp counts
    uint32_t scan_h[8], scan_t[8];      // warp totals of the two digit scans
};

template <int R>
__global__ void __launch_bounds__(kSortThreads, R == kSortMinRounds ? 2 : 1) k_sort_pass(
    int n, int pass, const uint64_t *__restrict kin, const uint32_t *__restrict vin,
    uint64_t *__restrict kout, uint32_t *__restrict vout, const IterCounters *__restrict ctr,
    uint32_t *__restrict counts, int ntiles, const DevState *__restrict st) {
    constexpr int kTile = kSortThreads * R;
    constexpr int kChunk = kTile / kSortWarps;  // keys per warp
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SortSmem<R> &S = *reinterpret_cast<SortSmem<R> *>(smem_raw);
    if (st->err || st->poison) return;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int shift = 8 * pass;
    const int tile = blockIdx.x;
    const int base = tile * kTile + wid * kChunk;
    const unsigned lt_mask = (1u << lane) - 1u;

    // 1. the warp's chunk (all loads in flight) ...
    uint64_t k[R];
    uint32_t v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int idx = base + r * 32 + lane;
        k[r] = idx < n ? kin[idx] : 0ull;
        v[r] = idx < n ? vin[idx] : 0u;
    }
    // ... and this tile's prefix per digit: the counts of all earlier tiles,
    // summed by 4 threads per digit with 8 loads in flight each
    uint32_t prefix_part;
    {
        const uint32_t *cp = counts + (size_t)pass * ntiles * 256 + (threadIdx.x & 255);
        uint32_t a[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int t = threadIdx.x >> 8; t < tile; t += 4 * 8) {
#pragma unroll
            for (int j = 0; j < 8; ++j)
                if (t + 4 * j < tile) a[j] += __ldcg(cp + (size_t)(t + 4 * j) * 256);
        }
        prefix_part = ((a[0] + a[1]) + (a[2] + a[3])) + ((a[4] + a[5]) + (a[6] + a[7]));
    }
    for (int j = threadIdx.x; j < kSortWarps * 256; j += kSortThreads) (&S.whist[0][0])[j] = 0;
    S.part[threadIdx.x >> 8][threadIdx.x & 255] = prefix_part;
    __syncthreads();

    // 2. rank round by round; an invalid lane gets a 9th digit bit so that it
    //    shares no valid lane's digit
    uint32_t rank[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const bool valid = base + r * 32 + lane < n;
        const uint32_t d = (uint32_t)(k[r] >> shift) & 255u;
        unsigned peers = __ballot_sync(kFull, valid);
        if (!valid) peers = ~peers;
#pragma unroll
        for (int b = 0; b < 8; ++b) {
            const bool bit = (d >> b) & 1u;
            const unsigned m = __ballot_sync(kFull, bit);
            peers &= bit ? m : ~m;
        }
        uint32_t before = 0;
        if (valid) before = S.whist[wid][d];
        rank[r] = before + __popc(peers & lt_mask);
        __syncwarp();
        if (valid && (peers & lt_mask) == 0) S.whist[wid][d] = before + __popc(peers);
        __syncwarp();
    }
    __syncthreads();

    // 3. per digit: exclusive offsets across the 32 warps (4 threads per
    //    digit, 8 warps each), the tile's digit counts, the prefix over the
    //    earlier tiles and the global start
    const int dg = threadIdx.x & 255, qt = threadIdx.x >> 8;
    {
        uint32_t q = 0;
#pragma unroll
        for (int w = 0; w < 8; ++w) q += S.whist[qt * 8 + w][dg];
        S.qsum[qt][dg] = q;
    }
    __syncthreads();
    uint32_t tile_count = 0, hist_d = 0, prefix = 0;
    {
        uint32_t run = 0;
#pragma unroll
        for (int q = 0; q < kQuarters; ++q) {
            const uint32_t c = S.qsum[q][dg];
            if (q < qt) run += c;
            tile_count += c;
        }
#pragma unroll
        for (int w = 0; w < 8; ++w) {
            const uint32_t c = S.whist[qt * 8 + w][dg];
            S.whist[qt * 8 + w][dg] = run;
            run += c;
        }
    }
    // both digit scans (global histogram, tile counts) in warps 0..7
    const bool digit_thread = threadIdx.x < 256;
    uint32_t inc_h = 0, inc_t = 0;
    if (digit_thread) {
        prefix = (S.part[0][dg] + S.part[1][dg]) + (S.part[2][dg] + S.part[3][dg]);
        hist_d = ctr->hist[pass][dg];
        inc_h = hist_d;
        inc_t = tile_count;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t th = __shfl_up_sync(kFull, inc_h, o);
            const uint32_t tt = __shfl_up_sync(kFull, inc_t, o);
            if (lane >= o) {
                inc_h += th;
                inc_t += tt;
            }
        }
        if (lane == 31) {
            S.scan_h[wid] = inc_h;
            S.scan_t[wid] = inc_t;
        }
    }
    __syncthreads();
    if (digit_thread) {
        uint32_t bh = 0, bt = 0;
        for (int w = 0; w < wid; ++w) {
            bh += S.scan_h[w];
            bt += S.scan_t[w];
        }
        S.gbase[dg] = bh + inc_h - hist_d + prefix;
        S.tile_off[dg] = bt + inc_t - tile_count;
    }
    __syncthreads();

    // 4. regroup by digit in shared memory, then write digit runs and count
    //    the next pass's digits per output tile
#pragma unroll
    for (int r = 0; r < R; ++r) {
        if (base + r * 32 + lane < n) {
            const uint32_t dd = (uint32_t)(k[r] >> shift) & 255u;
            const uint32_t p = S.tile_off[dd] + S.whist[wid][dd] + rank[r];
            S.keys[p] = k[r];
            S.vals[p] = v[r];
        }
    }
    __syncthreads();
    const int tile_n = min(kTile, n - tile * kTile);
    uint32_t *next = pass < 7 ? counts + (size_t)(pass + 1) * ntiles * 256 : nullptr;
    for (int j = threadIdx.x; j < tile_n; j += kSortThreads) {
        const uint64_t key = S.keys[j];
        const uint32_t dd = (uint32_t)(key >> shift) & 255u;
        const uint32_t out = S.gbase[dd] + (uint32_t)j - S.tile_off[dd];
        kout[out] = key;
        vout[out] = S.vals[j];
        if (next)
            atomicAdd(&next[(size_t)(out / kTile) * 256 + ((uint32_t)(key >> (shift + 8)) & 255u)], 1u);
    }
}

// After a sort that skipped the lowest `first` digits, keys equal in the
// sorted digits form runs in input order.  Sorting each run by the full key,
// stably, gives exactly the order of the full sort.  A run longer than
// kMaxRun asks for the iteration again with every digit (resort + poison: the
// iteration's later kernels skip their work and the host replays it).
__global__ void __launch_bounds__(256) k_fix_low(int n, int first, uint64_t *__restrict keys,
                                                 uint32_t *__restrict vals, DevState *st) {
    if (st->err || st->poison) return;
    const int low = 8 * first;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k + 1 < n;
         k += gridDim.x * blockDim.x) {
        const uint64_t hk = keys[k] >> low;
        if ((keys[k + 1] >> low) != hk || (k > 0 && (keys[k - 1] >> low) == hk)) continue;
        int len = 2;
        while (k + len < n && (keys[k + len] >> low) == hk && len <= kMaxRun) ++len;
        if (len > kMaxRun) {
            atomicExch(&st->resort, 1);
            atomicExch(&st->poison, 1);
            continue;
        }
        uint64_t *kr = keys + k;
        uint32_t *vr = vals + k;
        for (int a = 1; a < len; ++a) {  // insertion sort, stable
            const uint64_t ka = kr[a];
            const uint32_t va = vr[a];
            int j = a - 1;
            while (j >= 0 && kr[j] > ka) {
                kr[j + 1] = kr[j];
                vr[j + 1] = vr[j];
                --j;
            }
            kr[j + 1] = ka;
            vr[j + 1] = va;
        }
    }
}

template <int R>
void launch_passes(const Buffers &b, cudaStream_t s) {
    const int tiles = sort_tiles(b.n, R);
    for (int pass = b.sort_first; pass < 8; ++pass) {
        const int src = pass & 1, dst = src ^ 1;
        k_sort_pass<R><<<tiles, kSortThreads, sizeof(SortSmem<R>), s>>>(
            b.n, pass, b.keys[src], b.vals[src], b.keys[dst], b.vals[dst], b.ctr, b.sort_counts,
            tiles, b.st);
    }
}

}  // namespace

void sort_set_smem_attr() {
    cudaFuncSetAttribute(k_sort_pass<4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sizeof(SortSmem<4>));
    cudaFuncSetAttribute(k_sort_pass<5>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sizeof(SortSmem<5>));
    cudaFuncSetAttribute(k_sort_pass<6>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sizeof(SortSmem<6>));
}

void launch_fix_low(const Buffers &b, int nsm, cudaStream_t s) {
    if (b.sort_first <= 0 || b.n < 2) return;
    int grid = (b.n + 255) / 256;
    grid = grid > nsm * 8 ? nsm * 8 : grid;
    k_fix_low<<<grid, 256, 0, s>>>(b.n, b.sort_first, b.keys[0], b.vals[0], b.st);
}

void launch_sort(const Buffers &b, cudaStream_t s) {
    switch (b.sort_rounds) {
        case 5: launch_passes<5>(b, s); break;
        case 6: launch_passes<6>(b, s); break;
        default: launch_passes<4>(b, s); break;
    }
}

}  // namespace fa2
