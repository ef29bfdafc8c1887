// fa2_render.cu -- headless rendering of a layout on the GPU: the picture
// GraphLayout::writeToPNG draws (src/RPGraphLayout.cpp:170-207), computed as
// coverage counts instead of sequential blends.
//
// The reference blends every node disc and edge line in black onto a white
// image (pngwriter's filledcircle_blend / line_blend).  Blending black at
// opacity a scales a pixel by (1 - a), so the final pixel is the product of
// (1 - a) over every plot that covers it, whatever the order: the image is
// (1 - a_node)^(discs covering it) x (1 - a_edge)^(lines covering it), and 0
// once any plot with a >= 1 covers it (the blend clamps at black).  The GPU
// counts coverage with integer atomics (order-free, so deterministic), then
// shades.  pngwriter itself is not part of the reference's sources (an empty
// submodule), so the pixel rules below are this engine's:
//   * coordinates as the reference computes them, truncated to int;
//     pixel (x, y) is 1-based with y up, inside [1, w] x [1, h];
//   * a disc is every pixel within distance 3 of the centre;
//   * a line is the Bresenham sequence between its integer end points, both
//     ends included, each pixel once.
#include <cuda_runtime.h>
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>

#include "../../include/fa2b200.h"

namespace {

constexpr int kDiscRadius = 3;  // src/RPGraphLayout.cpp:193

struct Frame {
    float minx, miny, xscale, yscale;
    int w, h;
};

__device__ __forceinline__ void plot(const Frame &F, int x, int y, uint32_t *count) {
    if (x < 1 || x > F.w || y < 1 || y > F.h) return;
    const size_t row = (size_t)(F.h - y), col = (size_t)(x - 1);
    atomicAdd(&count[row * F.w + col], 1u);
}

__device__ __forceinline__ int to_px(float v, float lo, float scale) {
    return (int)((v - lo) * scale);  // float -> int truncation, as the int parameters take it
}

__global__ void k_discs(uint32_t n, const float2 *__restrict xy, Frame F, uint32_t *count) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float2 p = xy[i];
        const int cx = to_px(p.x, F.minx, F.xscale), cy = to_px(p.y, F.miny, F.yscale);
        for (int dy = -kDiscRadius; dy <= kDiscRadius; ++dy)
            for (int dx = -kDiscRadius; dx <= kDiscRadius; ++dx)
                if (dx * dx + dy * dy <= kDiscRadius * kDiscRadius) plot(F, cx + dx, cy + dy, count);
    }
}

// One warp per edge: lane j plots steps j, j + 32, ... of the line.  Step t
// of a line with major extent D and minor extent d (both >= 0) sits at
// major + t and minor + floor((2 t d + D) / (2 D)), each with its sign.
__global__ void k_lines(uint64_t m, const uint32_t *__restrict src, const uint32_t *__restrict dst,
                        const float2 *__restrict xy, Frame F, uint32_t *count) {
    const int lane = threadIdx.x & 31;
    const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t e = warp; e < m; e += warps) {
        const float2 a = xy[src[e]], b = xy[dst[e]];
        const int x1 = to_px(a.x, F.minx, F.xscale), y1 = to_px(a.y, F.miny, F.yscale);
        const int x2 = to_px(b.x, F.minx, F.xscale), y2 = to_px(b.y, F.miny, F.yscale);
        const long long ax = llabs((long long)x2 - x1), ay = llabs((long long)y2 - y1);
        const int sx = x2 >= x1 ? 1 : -1, sy = y2 >= y1 ? 1 : -1;
        const bool xmajor = ax >= ay;
        const long long D = xmajor ? ax : ay, d = xmajor ? ay : ax;
        for (long long t = lane; t <= D; t += 32) {
            const long long mi = D ? (2 * t * d + D) / (2 * D) : 0;
            const int x = xmajor ? x1 + (int)(sx * t) : x1 + (int)(sx * mi);
            const int y = xmajor ? y1 + (int)(sy * mi) : y1 + (int)(sy * t);
            plot(F, x, y, count);
        }
    }
}

__global__ void k_shade(size_t pixels, const uint32_t *__restrict discs,
                        const uint32_t *__restrict lines, float a_node, float a_edge,
                        uint8_t *__restrict rgb) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < pixels;
         i += (size_t)gridDim.x * blockDim.x) {
        const uint32_t cn = discs[i], ce = lines[i];
        double v;
        if ((cn && a_node >= 1.0f) || (ce && a_edge >= 1.0f))
            v = 0.0;
        else
            v = pow(1.0 - (double)a_node, (double)cn) * pow(1.0 - (double)a_edge, (double)ce);
        const uint8_t c = (uint8_t)fmin(255.0, floor(v * 255.0 + 0.5));
        rgb[3 * i] = c;
        rgb[3 * i + 1] = c;
        rgb[3 * i + 2] = c;
    }
}

}  // namespace

extern "C" int fa2_render_rgb(uint32_t num_nodes, uint64_t num_edges, const uint32_t *sources,
                              const uint32_t *targets, const float *xy, int32_t image_w,
                              int32_t image_h, int32_t device, uint8_t *rgb) {
    if (image_w <= 0 || image_h <= 0 || !rgb || (num_nodes && !xy) ||
        (num_edges && (!sources || !targets)))
        return FA2_ERR_INVALID_ARGUMENT;
    for (uint64_t e = 0; e < num_edges; ++e)
        if (sources[e] >= num_nodes || targets[e] >= num_nodes) return FA2_ERR_INVALID_ARGUMENT;
    const size_t pixels = (size_t)image_w * (size_t)image_h;
    if (pixels > (1ull << 31)) return FA2_ERR_TOO_LARGE;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
        return FA2_ERR_NO_DEVICE;
    if (cudaSetDevice(device) != cudaSuccess) return FA2_ERR_CUDA;

    // the frame, in the reference's float/double arithmetic (src/RPGraphLayout.cpp:173-186,
    // getCenter :141-146, getXRange :96-99)
    float mnx = FLT_MAX, mxx = -FLT_MAX, mny = FLT_MAX, mxy = -FLT_MAX;
    for (uint32_t i = 0; i < num_nodes; ++i) {
        mnx = fminf(mnx, xy[2 * i]);
        mxx = fmaxf(mxx, xy[2 * i]);
        mny = fminf(mny, xy[2 * i + 1]);
        mxy = fmaxf(mxy, xy[2 * i + 1]);
    }
    const float x_range = mxx - mnx, y_range = mxy - mny;
    const float x_center = mnx + x_range / 2.0, y_center = mny + y_range / 2.0;
    Frame F;
    F.minx = x_center - x_range / 2.0;
    F.miny = y_center - y_range / 2.0;
    F.xscale = image_w / x_range;
    F.yscale = image_h / y_range;
    F.w = image_w;
    F.h = image_h;
    const float a_node = 10000.0 / num_nodes;
    const float a_edge = 100000.0 / num_edges;

    float2 *d_xy = nullptr;
    uint32_t *d_s = nullptr, *d_t = nullptr, *d_cn = nullptr, *d_ce = nullptr;
    uint8_t *d_rgb = nullptr;
    int status = FA2_OK;
    cudaStream_t st = nullptr;
    auto ck = [&](cudaError_t e) {
        if (e != cudaSuccess && status == FA2_OK)
            status = e == cudaErrorMemoryAllocation ? FA2_ERR_OUT_OF_MEMORY : FA2_ERR_CUDA;
        return status == FA2_OK;
    };
    if (ck(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking)) &&
        ck(cudaMalloc(&d_xy, 8 * (size_t)(num_nodes ? num_nodes : 1))) &&
        ck(cudaMalloc(&d_s, 4 * (size_t)(num_edges ? num_edges : 1))) &&
        ck(cudaMalloc(&d_t, 4 * (size_t)(num_edges ? num_edges : 1))) &&
        ck(cudaMalloc(&d_cn, 4 * pixels)) && ck(cudaMalloc(&d_ce, 4 * pixels)) &&
        ck(cudaMalloc(&d_rgb, 3 * pixels)) &&
        ck(cudaMemcpyAsync(d_xy, xy, 8 * (size_t)num_nodes, cudaMemcpyHostToDevice, st)) &&
        ck(cudaMemcpyAsync(d_s, sources, 4 * (size_t)num_edges, cudaMemcpyHostToDevice, st)) &&
        ck(cudaMemcpyAsync(d_t, targets, 4 * (size_t)num_edges, cudaMemcpyHostToDevice, st)) &&
        ck(cudaMemsetAsync(d_cn, 0, 4 * pixels, st)) && ck(cudaMemsetAsync(d_ce, 0, 4 * pixels, st))) {
        if (num_nodes) k_discs<<<1024, 256, 0, st>>>(num_nodes, d_xy, F, d_cn);
        if (num_edges) k_lines<<<2048, 256, 0, st>>>(num_edges, d_s, d_t, d_xy, F, d_ce);
        k_shade<<<2048, 256, 0, st>>>(pixels, d_cn, d_ce, a_node, a_edge, d_rgb);
        if (ck(cudaGetLastError()))
            ck(cudaMemcpyAsync(rgb, d_rgb, 3 * pixels, cudaMemcpyDeviceToHost, st));
        ck(cudaStreamSynchronize(st));
    }
    cudaFree(d_xy);
    cudaFree(d_s);
    cudaFree(d_t);
    cudaFree(d_cn);
    cudaFree(d_ce);
    cudaFree(d_rgb);
    if (st) cudaStreamDestroy(st);
    return status;
}
