// The two ends of vx-vision's depth chain around SGM: the RGBA -> gray ingest
// conversion (ColorConvert::rgba_to_gray, vx-vision/shaders/ColorConvert.metal:
// 21-32) and the unprojection of a depth map to a point cloud
// (DepthToCloud::compute, vx-vision/shaders/DepthToCloud.metal:30-70).
//
// rgba_to_gray: gray = 0.299 r + 0.587 g + 0.114 b on the unorm values (byte /
// 255, single precision, that operation order, no contraction), stored as an
// 8-bit unorm (clamped to [0, 1], times 255, rounded to nearest even). One
// thread per 4 pixels: four 4-byte texel loads (a warp reads 512 contiguous
// bytes), one 4-byte store when aligned. HBM-bound: 5 bytes a pixel.
//
// depth_to_cloud: for each pixel, d = depth * depth_scale; pixels with
// d < min_depth or d > max_depth are dropped (NaN passes both tests, as in the
// shader); the others give X = (x - cx) * d / fx, Y = (y - cy) * d / fy, Z = d
// (IEEE single precision, the shader's order), colour (r, g, b, 255) from an
// RGBA8 image, (v, 0, 0, 255) from a U8 one, white without one, normal 0. The
// shader appends points with an atomic counter (unspecified order); here they
// come out in row-major pixel order, the first max_points of them, which is one
// of the shader's possible outputs: a count kernel per 1024-pixel tile, then
// an emit kernel whose CTA t sums the counts of tiles before t (no waiting on
// other CTAs), ranks its valid pixels with a block scan and writes the 36-byte
// records. The last CTA writes the number of pixels that passed.
#include <cuda_runtime.h>

#include "kernels.cuh"
#include "launch.hpp"

namespace vxsgm {

namespace {

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ uint32_t gray_of(uint32_t rgba, const float* __restrict__ unorm) {
    const float r = unorm[rgba & 0xFFu], g = unorm[(rgba >> 8) & 0xFFu], b = unorm[(rgba >> 16) & 0xFFu];
    const float v = __fadd_rn(__fadd_rn(__fmul_rn(0.299f, r), __fmul_rn(0.587f, g)), __fmul_rn(0.114f, b));
    return (uint32_t)__float2int_rn(__fmul_rn(fminf(fmaxf(v, 0.0f), 1.0f), 255.0f));
}

__global__ void __launch_bounds__(256)
rgba_to_gray_kernel(const uint8_t* __restrict__ in, size_t in_pitch, uint8_t* __restrict__ out, size_t out_pitch,
                    int W, int H) {
    __shared__ float unorm[256];      // byte / 255 (the texel read of an 8-bit unorm channel)
    unorm[threadIdx.x] = __fdiv_rn((float)threadIdx.x, 255.0f);
    __syncthreads();
    const int quads = (W + 3) / 4;
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= (long long)quads * H) return;
    const int y = (int)(q / quads), x = (int)(q % quads) * 4;
    const uint32_t* src = reinterpret_cast<const uint32_t*>(in + (size_t)y * in_pitch) + x;
    uint8_t* dst = out + (size_t)y * out_pitch + x;
    const int n = min(4, W - x);
    uint32_t g[4] = {0u, 0u, 0u, 0u};
#pragma unroll
    for (int i = 0; i < 4; ++i)
        if (i < n) g[i] = gray_of(__ldg(src + i), unorm);
    if (n == 4 && (reinterpret_cast<uintptr_t>(dst) & 3u) == 0) {
        *reinterpret_cast<uint32_t*>(dst) = g[0] | (g[1] << 8) | (g[2] << 16) | (g[3] << 24);
    } else {
        for (int i = 0; i < n; ++i) dst[i] = (uint8_t)g[i];
    }
}

constexpr int kCloudThreads = 256;
constexpr int kCloudPerThread = 4;
constexpr int kCloudTile = kCloudThreads * kCloudPerThread;   // pixels of one tile (row-major run)

struct CloudArgs {
    const float* depth;
    size_t depth_pitch;       // bytes
    const uint8_t* color;     // nullptr: white
    size_t color_pitch;
    int color_rgba;           // 1: RGBA8, 0: U8
    int W, H;
    float fx, fy, cx, cy, min_depth, max_depth, depth_scale;
    uint32_t max_points;
};

// The pixel's depth after scaling and whether it passes the range test.
__device__ __forceinline__ bool cloud_valid(const CloudArgs& a, long long p, float& d) {
    if (p >= (long long)a.W * a.H) return false;
    const int y = (int)(p / a.W), x = (int)(p % a.W);
    d = __fmul_rn(__ldg(reinterpret_cast<const float*>(reinterpret_cast<const char*>(a.depth) + (size_t)y * a.depth_pitch) + x),
                  a.depth_scale);
    return !(d < a.min_depth || d > a.max_depth);
}

__device__ __forceinline__ uint32_t block_sum(uint32_t v, uint32_t* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    uint32_t s = 0;
#pragma unroll
    for (int w = 0; w < kCloudThreads / 32; ++w) s += red[w];
    __syncthreads();
    return s;
}

__global__ void __launch_bounds__(kCloudThreads)
cloud_count_kernel(const CloudArgs a, uint32_t* __restrict__ tile_counts) {
    __shared__ uint32_t red[kCloudThreads / 32];
    uint32_t n = 0;
#pragma unroll
    for (int k = 0; k < kCloudPerThread; ++k) {
        float d;
        n += cloud_valid(a, (long long)blockIdx.x * kCloudTile + k * kCloudThreads + threadIdx.x, d) ? 1u : 0u;
    }
    n = block_sum(n, red);
    if (threadIdx.x == 0) tile_counts[blockIdx.x] = n;
}

__global__ void __launch_bounds__(kCloudThreads)
cloud_emit_kernel(const CloudArgs a, const uint32_t* __restrict__ tile_counts, int tiles,
                  float* __restrict__ points, uint32_t* __restrict__ count) {
    __shared__ uint32_t red[kCloudThreads / 32];
    __shared__ uint32_t warp_base[kCloudThreads / 32];
    // Points of the tiles before this one.
    uint32_t before = 0;
    for (int t = threadIdx.x; t < (int)blockIdx.x; t += kCloudThreads) before += tile_counts[t];
    uint32_t base = block_sum(before, red);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int k = 0; k < kCloudPerThread; ++k) {
        const long long p = (long long)blockIdx.x * kCloudTile + k * kCloudThreads + threadIdx.x;
        float d = 0.0f;
        const bool v = cloud_valid(a, p, d);
        // Rank among this round's 256 pixels (pixel order = thread order).
        const unsigned bal = __ballot_sync(kFull, v);
        if (lane == 0) warp_base[warp] = __popc(bal);
        __syncthreads();
        uint32_t off = base, total = 0;
#pragma unroll
        for (int w = 0; w < kCloudThreads / 32; ++w) {
            off += w < warp ? warp_base[w] : 0u;
            total += warp_base[w];
        }
        __syncthreads();
        const uint32_t slot = off + __popc(bal & ((1u << lane) - 1u));
        if (v && slot < a.max_points) {
            const int y = (int)(p / a.W), x = (int)(p % a.W);
            const float X = __fdiv_rn(__fmul_rn(__fsub_rn((float)x, a.cx), d), a.fx);
            const float Y = __fdiv_rn(__fmul_rn(__fsub_rn((float)y, a.cy), d), a.fy);
            uint32_t rgba = 0xFFFFFFFFu;
            if (a.color) {
                const uint8_t* row = a.color + (size_t)y * a.color_pitch;
                rgba = a.color_rgba ? (__ldg(reinterpret_cast<const uint32_t*>(row) + x) | 0xFF000000u)
                                    : ((uint32_t)__ldg(row + x) | 0xFF000000u);
            }
            float* r = points + (size_t)slot * 9;   // 36-byte GpuPoint3D records
            r[0] = X;
            r[1] = Y;
            r[2] = d;
            r[3] = 0.0f;
            reinterpret_cast<uint32_t*>(r)[4] = rgba;
            r[5] = 0.0f;
            r[6] = 0.0f;
            r[7] = 0.0f;
            r[8] = 0.0f;
        }
        base += total;
    }
    if (blockIdx.x == tiles - 1 && threadIdx.x == 0) *count = base;
}

}  // namespace

cudaError_t launch_rgba_to_gray(const uint8_t* in, size_t in_pitch, uint8_t* out, size_t out_pitch, int W, int H,
                                cudaStream_t stream) {
    const long long quads = (long long)((W + 3) / 4) * H;
    if (quads == 0) return cudaSuccess;
    count_launch();
    rgba_to_gray_kernel<<<(unsigned)((quads + 255) / 256), 256, 0, stream>>>(in, in_pitch, out, out_pitch, W, H);
    return cudaGetLastError();
}

int depth_to_cloud_tiles(int W, int H) { return (int)(((long long)W * H + kCloudTile - 1) / kCloudTile); }

cudaError_t launch_depth_to_cloud(const float* depth, size_t depth_pitch, const uint8_t* color, size_t color_pitch,
                                  bool color_rgba, int W, int H, float fx, float fy, float cx, float cy,
                                  float min_depth, float max_depth, float depth_scale, uint32_t max_points,
                                  uint32_t* tile_counts, float* points, uint32_t* count, cudaStream_t stream) {
    const int tiles = depth_to_cloud_tiles(W, H);
    if (tiles == 0) return cudaSuccess;
    CloudArgs a{depth, depth_pitch, color, color_pitch, color_rgba ? 1 : 0, W, H, fx, fy, cx, cy,
                min_depth, max_depth, depth_scale, max_points};
    count_launch(2);
    cloud_count_kernel<<<tiles, kCloudThreads, 0, stream>>>(a, tile_counts);
    cloud_emit_kernel<<<tiles, kCloudThreads, 0, stream>>>(a, tile_counts, tiles, points, count);
    return cudaGetLastError();
}

}  // namespace vxsgm
