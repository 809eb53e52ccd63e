// Depth-map post-filters (vx-vision's DepthFilter: kernels/depth_filter.rs,
// shaders/DepthFilter.metal), the step after WTA in vx-vision's depth chain:
// a median filter over the valid (> 0) values of a window, and an
// edge-preserving bilateral filter.
//
// Semantics (DepthFilter.metal:84-120, depth_median): the valid values of the
// (2r+1)^2 window with clamped coordinates, in raster order; the output is the
// element at index count/2 of their ascending order (the upper middle for an
// even count), or 0 when none is valid. Invalid SGM pixels (LR check, value
// -1) are therefore left out. (DepthFilter.metal:20-66, depth_bilateral): a
// centre <= 0 gives 0; otherwise the mean of the valid neighbours weighted by
// exp(-(dx^2+dy^2) / (2 ss^2)) * exp(-(n-c)^2 / (2 sd^2)), or the centre when
// the weights sum to at most 1e-8; single-precision arithmetic in the shader's
// order, without fused multiply-adds (so only expf may differ from a host's).
//
// Mapping: one thread per output pixel of a 32x8 tile; the tile and its apron
// (clamped coordinates) are staged in shared memory once per CTA. Median: the
// window's values go to registers with invalid ones as +inf, and the output is
// the value of rank count/2 (rank = smaller values + equal values earlier in
// raster order), which equals the shader's sorted pick without a sort.
// Bilateral: the spatial weights of the window are computed once per CTA.
#include <cuda_runtime.h>

#include <cmath>

#include "launch.hpp"

namespace vxsgm {

namespace {

constexpr int kTileW = 32, kTileH = 8;

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// Stages the tile of the CTA and its apron of r pixels (clamped) into s (row
// stride tw = 32 + 2r).
__device__ __forceinline__ void stage_tile(const float* __restrict__ in, size_t pitch, int W, int H, int r,
                                           float* __restrict__ s) {
    const int tw = kTileW + 2 * r, th = kTileH + 2 * r;
    const int x0 = blockIdx.x * kTileW - r, y0 = blockIdx.y * kTileH - r;
    for (int i = threadIdx.y * kTileW + threadIdx.x; i < tw * th; i += kTileW * kTileH) {
        const int ty = i / tw, tx = i - ty * tw;
        const int gx = clampi(x0 + tx, 0, W - 1), gy = clampi(y0 + ty, 0, H - 1);
        s[i] = *reinterpret_cast<const float*>(reinterpret_cast<const char*>(in) + (size_t)gy * pitch +
                                               (size_t)gx * sizeof(float));
    }
}

// Median for a compile-time radius R (window in registers, unrolled ranks).
template <int R>
__global__ void __launch_bounds__(kTileW * kTileH)
median_kernel(const float* __restrict__ in, size_t in_pitch, float* __restrict__ out, size_t out_pitch, int W,
              int H) {
    constexpr int N = (2 * R + 1) * (2 * R + 1);
    constexpr int TW = kTileW + 2 * R;
    __shared__ float s[(kTileH + 2 * R) * (kTileW + 2 * R)];
    stage_tile(in, in_pitch, W, H, R, s);
    __syncthreads();
    const int x = blockIdx.x * kTileW + threadIdx.x, y = blockIdx.y * kTileH + threadIdx.y;
    if (x >= W || y >= H) return;
    float v[N];
    int count = 0;
#pragma unroll
    for (int i = 0; i < N; ++i) {
        const float d = s[(threadIdx.y + i / (2 * R + 1)) * TW + threadIdx.x + i % (2 * R + 1)];
        const bool ok = d > 0.0f;
        v[i] = ok ? d : INFINITY;
        count += ok ? 1 : 0;
    }
    const int k = count / 2;
    float r = 0.0f;
#pragma unroll
    for (int i = 0; i < N; ++i) {
        int rank = 0;
#pragma unroll
        for (int j = 0; j < N; ++j) rank += (v[j] < v[i] || (j < i && v[j] == v[i])) ? 1 : 0;
        if (rank == k) r = v[i];
    }
    if (count == 0) r = 0.0f;
    *reinterpret_cast<float*>(reinterpret_cast<char*>(out) + (size_t)y * out_pitch + (size_t)x * sizeof(float)) = r;
}

// Median for radius 3..5 (window read from shared memory in loops).
__global__ void __launch_bounds__(kTileW * kTileH)
median_kernel_large(const float* __restrict__ in, size_t in_pitch, float* __restrict__ out, size_t out_pitch,
                    int W, int H, int R) {
    extern __shared__ float s[];
    stage_tile(in, in_pitch, W, H, R, s);
    __syncthreads();
    const int x = blockIdx.x * kTileW + threadIdx.x, y = blockIdx.y * kTileH + threadIdx.y;
    if (x >= W || y >= H) return;
    const int TW = kTileW + 2 * R, n = 2 * R + 1, N = n * n;
    auto val = [&](int i) {
        const float d = s[(threadIdx.y + i / n) * TW + threadIdx.x + i % n];
        return d > 0.0f ? d : INFINITY;
    };
    int count = 0;
    for (int i = 0; i < N; ++i) count += s[(threadIdx.y + i / n) * TW + threadIdx.x + i % n] > 0.0f ? 1 : 0;
    const int k = count / 2;
    float r = 0.0f;
    for (int i = 0; i < N && count > 0; ++i) {
        const float vi = val(i);
        int rank = 0;
        for (int j = 0; j < N; ++j) {
            const float vj = val(j);
            rank += (vj < vi || (j < i && vj == vi)) ? 1 : 0;
        }
        if (rank == k) {
            r = vi;
            break;
        }
    }
    *reinterpret_cast<float*>(reinterpret_cast<char*>(out) + (size_t)y * out_pitch + (size_t)x * sizeof(float)) = r;
}

__global__ void __launch_bounds__(kTileW * kTileH)
bilateral_kernel(const float* __restrict__ in, size_t in_pitch, float* __restrict__ out, size_t out_pitch, int W,
                 int H, int R, float sigma_s, float sigma_d) {
    extern __shared__ float s[];
    const int n = 2 * R + 1, TW = kTileW + 2 * R;
    float* ws = s + (kTileH + 2 * R) * TW;      // spatial weights, n*n
    stage_tile(in, in_pitch, W, H, R, s);
    const float inv_2ss = __fdiv_rn(1.0f, __fmul_rn(__fmul_rn(2.0f, sigma_s), sigma_s));
    const float inv_2sd = __fdiv_rn(1.0f, __fmul_rn(__fmul_rn(2.0f, sigma_d), sigma_d));
    for (int i = threadIdx.y * kTileW + threadIdx.x; i < n * n; i += kTileW * kTileH) {
        const int dy = i / n - R, dx = i % n - R;
        ws[i] = expf(__fmul_rn(-(float)(dx * dx + dy * dy), inv_2ss));
    }
    __syncthreads();
    const int x = blockIdx.x * kTileW + threadIdx.x, y = blockIdx.y * kTileH + threadIdx.y;
    if (x >= W || y >= H) return;
    const float c = s[(threadIdx.y + R) * TW + threadIdx.x + R];
    float res = 0.0f;
    if (!(c <= 0.0f)) {
        float sum = 0.0f, wsum = 0.0f;
        for (int i = 0; i < n * n; ++i) {
            const float nb = s[(threadIdx.y + i / n) * TW + threadIdx.x + i % n];
            if (nb <= 0.0f) continue;
            const float diff = __fsub_rn(nb, c);
            const float wd = expf(__fmul_rn(__fmul_rn(-diff, diff), inv_2sd));
            const float wt = __fmul_rn(ws[i], wd);
            sum = __fadd_rn(sum, __fmul_rn(nb, wt));
            wsum = __fadd_rn(wsum, wt);
        }
        res = wsum > 1e-8f ? __fdiv_rn(sum, wsum) : c;
    }
    *reinterpret_cast<float*>(reinterpret_cast<char*>(out) + (size_t)y * out_pitch + (size_t)x * sizeof(float)) =
        res;
}

size_t tile_floats(int r) { return (size_t)(kTileH + 2 * r) * (kTileW + 2 * r); }

}  // namespace

cudaError_t launch_depth_median(const float* in, size_t in_pitch, float* out, size_t out_pitch, int W, int H,
                                int radius, cudaStream_t stream) {
    const dim3 block(kTileW, kTileH), grid((W + kTileW - 1) / kTileW, (H + kTileH - 1) / kTileH);
    count_launch();
    switch (radius) {
        case 0: median_kernel<0><<<grid, block, 0, stream>>>(in, in_pitch, out, out_pitch, W, H); break;
        case 1: median_kernel<1><<<grid, block, 0, stream>>>(in, in_pitch, out, out_pitch, W, H); break;
        case 2: median_kernel<2><<<grid, block, 0, stream>>>(in, in_pitch, out, out_pitch, W, H); break;
        default:
            median_kernel_large<<<grid, block, tile_floats(radius) * sizeof(float), stream>>>(
                in, in_pitch, out, out_pitch, W, H, radius);
    }
    return cudaGetLastError();
}

cudaError_t launch_depth_bilateral(const float* in, size_t in_pitch, float* out, size_t out_pitch, int W, int H,
                                   int radius, float sigma_s, float sigma_d, cudaStream_t stream) {
    const dim3 block(kTileW, kTileH), grid((W + kTileW - 1) / kTileW, (H + kTileH - 1) / kTileH);
    const size_t smem = (tile_floats(radius) + (size_t)(2 * radius + 1) * (2 * radius + 1)) * sizeof(float);
    count_launch();
    bilateral_kernel<<<grid, block, smem, stream>>>(in, in_pitch, out, out_pitch, W, H, radius, sigma_s, sigma_d);
    return cudaGetLastError();
}

size_t depth_bilateral_smem_bytes(int radius) {
    return (tile_floats(radius) + (size_t)(2 * radius + 1) * (2 * radius + 1)) * sizeof(float);
}

}  // namespace vxsgm
