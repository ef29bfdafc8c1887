// fa2_noalloc.cu -- fa2_repulsion_noalloc: the engine's Barnes-Hut repulsion
// (bounding box, Morton keys, radix sort, tree build, warp-vote traversal) run
// on device buffers the caller owns, with every piece of scratch taken from
// one static device array of fixed size.  No call allocates device or host
// memory, so callers whose allocator must not be touched at the point of the
// call (a fixed device-memory budget, a caching allocator owned by a host
// framework, a process that reserved the device's memory up front) can still
// evaluate the repulsion.  The kernels are the ones fa2_step launches; only
// where their scratch lives differs.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <mutex>

#include "../../include/fa2b200.h"
#include "fa2_internal.cuh"

namespace fa2 {

namespace {

constexpr uint32_t kMaxBodies = FA2_NOALLOC_MAX_BODIES;
// nodes of the quadtree: at most 33 per body (the bound fa2_create allocates)
// plus one spare slot
constexpr uint64_t kMaxNodes = 33ull * kMaxBodies + 64;
constexpr int kMaxSMs = 256;  // k_bbox runs 2 blocks per SM, k_displace is not run
constexpr int kMaxDevices = 64;

constexpr size_t up256(size_t x) { return (x + 255) & ~(size_t)255; }
constexpr int tiles_of(uint32_t n, int tile) { return (int)((n + tile - 1) / tile); }

// Byte offsets of the sub-buffers inside the static array, each on a
// 256-byte boundary.  The first region is the one cleared on every call.
constexpr size_t kZeroBytes = sizeof(IterCounters) +
                              4 * ((size_t)8 * tiles_of(kMaxBodies, kSortTileMin) * 256 +
                                   (size_t)tiles_of(kMaxBodies, kCountTile));
constexpr size_t kOffZero = 0;
constexpr size_t kOffSt = up256(kOffZero + kZeroBytes);
constexpr size_t kOffFag = up256(kOffSt + sizeof(DevState));
constexpr size_t kOffFprev = up256(kOffFag + 8ull * kMaxBodies);
constexpr size_t kOffRef = up256(kOffFprev + 8ull * kMaxBodies);
constexpr size_t kOffKeys0 = up256(kOffRef + 4ull * kMaxBodies);
constexpr size_t kOffKeys1 = up256(kOffKeys0 + 8ull * kMaxBodies);
constexpr size_t kOffVals0 = up256(kOffKeys1 + 8ull * kMaxBodies);
constexpr size_t kOffVals1 = up256(kOffVals0 + 4ull * kMaxBodies);
constexpr size_t kOffLcp = up256(kOffVals1 + 4ull * kMaxBodies);
constexpr size_t kOffGroup = up256(kOffLcp + 1ull * kMaxBodies);
constexpr size_t kOffBodyNode = up256(kOffGroup + 4ull * kMaxBodies);
constexpr size_t kOffNodes = up256(kOffBodyNode + 4ull * kMaxBodies);
constexpr size_t kOffOwner = up256(kOffNodes + 16ull * (kMaxNodes + 1));
constexpr size_t kOffPm = up256(kOffOwner + 4ull * kMaxNodes);
constexpr size_t kOffPxy = up256(kOffPm + 8ull * (kMaxBodies + 1));
constexpr size_t kOffLookback =
    up256(kOffPxy + 2ull * sizeof(__int128) * (kMaxBodies + 1));
constexpr size_t kOffWarp =
    up256(kOffLookback + sizeof(LookbackSums) * tiles_of(kMaxBodies, kCountTile));
constexpr size_t kOffBBox = up256(kOffWarp + 8ull * ((kMaxBodies + 31) / 32));
constexpr size_t kScratchBytes = up256(kOffBBox + 16ull * 4 * kMaxSMs);
static_assert(kScratchBytes < (7u << 20), "the static scratch is meant to stay near 6 MB");

// The scratch: one per device, in the library's device image.  Static device
// memory starts zeroed when the module is loaded.
__device__ __align__(256) unsigned char g_scratch[kScratchBytes];

// Error bit of this entry point: a mass that is not a whole number in
// [0, 2^24).  The tree sums masses as exact integers, which FA2's masses
// (degree + 1) always are.
constexpr int kErrMass = 1 << 8;

// Reference ids (the caller's indices) and the mass check.
__global__ void k_prepare(uint32_t n, const float *__restrict mass, uint32_t *__restrict ids,
                          DevState *st) {
    bool bad = false;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        ids[i] = i;
        const float m = mass[i];
        bad |= !(m >= 0.0f && m < 16777216.0f && m == truncf(m));
    }
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(&st->err, kErrMass);
}

struct DeviceSetup {
    bool ready;
    unsigned char *base;  // device address of g_scratch on this device
    int nsm;
    int trav_blocks;
};

std::mutex g_setup_mutex;
DeviceSetup g_setup[kMaxDevices];

int status_of(cudaError_t e) { return e == cudaSuccess ? FA2_OK : FA2_ERR_CUDA; }

// First call on a device: with that device current, look up the address of
// g_scratch and set the kernels' launch attributes.  Later calls reuse both.
int setup_device(int device, DeviceSetup *out) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    DeviceSetup &d = g_setup[device];
    if (d.ready) {
        *out = d;
        return FA2_OK;
    }
    cudaDeviceProp dp;
    if (cudaGetDeviceProperties(&dp, device) != cudaSuccess || dp.major < 10)
        return FA2_ERR_NO_DEVICE;
    if (dp.multiProcessorCount > kMaxSMs) return FA2_ERR_DEVICE_LIMIT;
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess) return status_of(e);
    sort_set_smem_attr();
    d.trav_blocks = dp.multiProcessorCount * traverse_blocks_per_sm();
    d.base = static_cast<unsigned char *>(p);
    d.nsm = dp.multiProcessorCount;
    d.ready = true;
    *out = d;
    return FA2_OK;
}

int run(const float *d_xy, const float *d_mass, uint32_t n, const fa2_params *prm,
        cudaStream_t s, float *d_force, const DeviceSetup &d) {
    unsigned char *base = d.base;
    Buffers b;
    memset(&b, 0, sizeof(b));
    b.n = (int)n;
    b.pos = reinterpret_cast<float2 *>(const_cast<float *>(d_xy));  // read only here
    b.mass = const_cast<float *>(d_mass);                            // read only here
    b.f = reinterpret_cast<float2 *>(d_force);
    b.fag = reinterpret_cast<float2 *>(base + kOffFag);
    b.fprev = reinterpret_cast<float2 *>(base + kOffFprev);
    b.ref_of = reinterpret_cast<const uint32_t *>(base + kOffRef);
    b.keys[0] = reinterpret_cast<uint64_t *>(base + kOffKeys0);
    b.keys[1] = reinterpret_cast<uint64_t *>(base + kOffKeys1);
    b.vals[0] = reinterpret_cast<uint32_t *>(base + kOffVals0);
    b.vals[1] = reinterpret_cast<uint32_t *>(base + kOffVals1);
    b.lcp = reinterpret_cast<int8_t *>(base + kOffLcp);
    b.group = reinterpret_cast<uint32_t *>(base + kOffGroup);
    b.body_node = reinterpret_cast<uint32_t *>(base + kOffBodyNode);
    b.nodes = reinterpret_cast<float4 *>(base + kOffNodes);
    b.owner = reinterpret_cast<uint32_t *>(base + kOffOwner);
    b.capacity = (uint32_t)kMaxNodes;
    b.pm = reinterpret_cast<long long *>(base + kOffPm);
    b.pxy = reinterpret_cast<__int128 *>(base + kOffPxy);
    b.lookback = reinterpret_cast<LookbackSums *>(base + kOffLookback);
    b.warp_partial = reinterpret_cast<float2 *>(base + kOffWarp);
    b.bbox_partial = reinterpret_cast<float4 *>(base + kOffBBox);
    b.st = reinterpret_cast<DevState *>(base + kOffSt);
    b.ctr = reinterpret_cast<IterCounters *>(base + kOffZero);
    b.sort_rounds = sort_rounds((int)n, d.nsm);
    const size_t sort_counts = (size_t)8 * sort_tiles(b.n, b.sort_rounds) * 256;
    b.sort_counts = reinterpret_cast<uint32_t *>(base + kOffZero + sizeof(IterCounters));
    b.count_status = b.sort_counts + sort_counts;
    const size_t zero_bytes = sizeof(IterCounters) + 4 * (sort_counts + count_tiles((int)n));

    Params kp{};  // every field: the kernels read all of them
    kp.k_r = prm->scale;
    kp.k_g = 0.0f;
    kp.itolsq = 1.0f / (prm->theta * prm->theta);  // src/RPForceAtlas2.cpp:47
    kp.epssq = prm->epssq;
    kp.strong_gravity = 0;
    kp.linlog = 0;
    kp.multipole = 1;
    kp.nsm = d.nsm;
    kp.overlap = 0;

    // Must start at zero on every call: the counters, histograms, per-tile
    // digit counts and look-back flags; the device scalars (error and
    // coincidence flags, interaction count); the gravity + attraction term
    // the traversal adds to the repulsion (zero here, so d_force receives the
    // repulsion alone).  The reference ids are the caller's indices.
    cudaError_t e = cudaMemsetAsync(b.ctr, 0, zero_bytes, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(b.st, 0, sizeof(DevState), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(b.fag, 0, (size_t)n * sizeof(float2), s);
    if (e != cudaSuccess) return status_of(e);
    // A launch error is read from the runtime's last-error slot.  An error
    // the caller left there before this call is not ours to report or to
    // clear, so launch errors are taken from the slot only if it was empty on
    // entry (otherwise a failed launch still shows in the stream wait below).
    const bool slot_was_clear = cudaPeekAtLastError() == cudaSuccess;
    k_prepare<<<(n + 255) / 256, 256, 0, s>>>(n, d_mass, const_cast<uint32_t *>(b.ref_of), b.st);
    launch_bbox(b, d.nsm * 2, s);
    launch_keys(b, d.nsm, s);
    launch_sort(b, s);
    launch_tree_count(b, false, s);
    launch_emit(b, d.nsm, s);
    launch_traverse(b, kp, d.trav_blocks, s);
    if (slot_was_clear) {
        e = cudaGetLastError();
        if (e != cudaSuccess) return status_of(e);
    }
    int flags[2] = {0, 0};  // DevState::poison, DevState::err (adjacent)
    static_assert(offsetof(DevState, err) == offsetof(DevState, poison) + sizeof(int),
                  "poison and err are read with one copy");
    e = cudaMemcpyAsync(flags, &b.st->poison, sizeof(flags), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return status_of(e);
    if (flags[1] & (kErrMass | kErrNonFinite)) return FA2_ERR_INVALID_ARGUMENT;
    if (flags[1]) return FA2_ERR_DEVICE_LIMIT;
    if (flags[0]) return FA2_ERR_INVALID_ARGUMENT;  // coincident bodies
    return FA2_OK;
}

}  // namespace

}  // namespace fa2

extern "C" int fa2_repulsion_noalloc(const float *d_xy, const float *d_mass, uint32_t n,
                                     const fa2_params *prm, void *stream, float *d_force) {
    using namespace fa2;
    if (!prm) return FA2_ERR_INVALID_ARGUMENT;
    if (n > kMaxBodies) return FA2_ERR_TOO_LARGE;
    if (prm->multipole < 1) return FA2_ERR_INVALID_ARGUMENT;
    if (!prm->use_barneshut || prm->multipole != 1) return FA2_ERR_UNSUPPORTED;
    if (!(prm->theta > 0.0f)) return FA2_ERR_INVALID_ARGUMENT;
    if (n == 0) return FA2_OK;
    if (!d_xy || !d_mass || !d_force || ((uintptr_t)d_xy & 7) || ((uintptr_t)d_force & 7) ||
        ((uintptr_t)d_mass & 3))
        return FA2_ERR_INVALID_ARGUMENT;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || prm->device < 0 || prm->device >= ndev ||
        prm->device >= kMaxDevices)
        return FA2_ERR_NO_DEVICE;
    int prev = 0;
    if (cudaGetDevice(&prev) != cudaSuccess) return FA2_ERR_CUDA;
    if (prev != prm->device && cudaSetDevice(prm->device) != cudaSuccess) return FA2_ERR_CUDA;
    DeviceSetup d;
    int s = setup_device(prm->device, &d);
    if (s == FA2_OK) s = run(d_xy, d_mass, n, prm, static_cast<cudaStream_t>(stream), d_force, d);
    if (prev != prm->device) cudaSetDevice(prev);
    return s;
}
