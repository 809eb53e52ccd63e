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
// order, without fused multiply-adds. The spatial weights use expf; the range
// weight, one per neighbour, the __expf intrinsic (a few ulp from expf, and
// Metal's fast-math exp is not exact either), so results agree with a host
// build to about 1e-6 relative.
//
// Mapping: one thread per output pixel of a 32x8 tile; the tile and its apron
// (clamped coordinates) are staged in shared memory once per CTA. Median: the
// window's values go to registers with invalid ones as +inf, and the output is
// the value of rank count/2 (rank = smaller values + equal values earlier in
// raster order), which equals the shader's sorted pick without a sort.
// Bilateral: the spatial weights of the window are computed once per CTA.
#include <cuda_runtime.h>

#include <cmath>
#include <utility>

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

// Batcher's odd-even merge sorting network restricted to N inputs (a
// comparator that would touch index >= N meets an implicit +inf and is a
// no-op, so it is left out), as a compile-time list of index pairs.
template <int N>
struct SortNet {
    int a[512] = {}, b[512] = {};
    int n = 0;
    constexpr SortNet() {
        for (int p = 1; p < N; p <<= 1)
            for (int k = p; k >= 1; k >>= 1)
                for (int j = k % p; j + k < N; j += 2 * k)
                    for (int i = 0; i < k; ++i)
                        if (i + j + k < N && (i + j) / (2 * p) == (i + j + k) / (2 * p)) {
                            a[n] = i + j;
                            b[n] = i + j + k;
                            ++n;
                        }
    }
};
template <int N>
constexpr SortNet<N> kSortNet{};

template <int A, int B, int N>
__device__ __forceinline__ void compare_exchange(uint32_t (&v)[N]) {
    const uint32_t x = v[A], y = v[B];
    v[A] = min(x, y);
    v[B] = max(x, y);
}

template <int N, int... I>
__device__ __forceinline__ void apply_net(uint32_t (&v)[N], std::integer_sequence<int, I...>) {
    (compare_exchange<kSortNet<N>.a[I], kSortNet<N>.b[I]>(v), ...);
}

// Sorts v ascending; every index is a template argument, so v stays in registers.
template <int N>
__device__ __forceinline__ void sort_network(uint32_t (&v)[N]) {
    apply_net<N>(v, std::make_integer_sequence<int, kSortNet<N>.n>{});
}

// Median for a compile-time radius R (window in registers). The values taken
// (> 0, +inf included) and the +inf standing in for invalid ones are positive
// floats, whose order is that of their bit patterns: the window is sorted as
// uint32 and the element of index count/2 is read (equal values have equal
// bits, so this is the shader's pick). Only indices <= N/2 are read, so the
// compiler drops the comparators that feed only the upper half.
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
    constexpr uint32_t kInf = 0x7F800000u;
    uint32_t v[N];
    int count = 0;
#pragma unroll
    for (int i = 0; i < N; ++i) {
        const float d = s[(threadIdx.y + i / (2 * R + 1)) * TW + threadIdx.x + i % (2 * R + 1)];
        const bool ok = d > 0.0f;
        v[i] = ok ? __float_as_uint(d) : kInf;
        count += ok ? 1 : 0;
    }
    sort_network<N>(v);
    const int k = count / 2;
    uint32_t pick = v[0];
#pragma unroll
    for (int i = 1; i <= N / 2; ++i) pick = k == i ? v[i] : pick;
    const float r = count == 0 ? 0.0f : __uint_as_float(pick);
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
    const int TW = kTileW + 2 * R, n = 2 * R + 1;
    const float* win = s + threadIdx.y * TW + threadIdx.x;  // the window's top-left value
    // Values in raster order: element i = (i / n, i % n), walked row by row.
    auto val = [&](int dy, int dx) {
        const float d = win[dy * TW + dx];
        return d > 0.0f ? d : INFINITY;
    };
    int count = 0;
    for (int dy = 0; dy < n; ++dy)
        for (int dx = 0; dx < n; ++dx) count += win[dy * TW + dx] > 0.0f ? 1 : 0;
    const int k = count / 2;
    float r = 0.0f;
    bool found = count == 0;
    for (int iy = 0; iy < n && !found; ++iy)
        for (int ix = 0; ix < n && !found; ++ix) {
            const float vi = val(iy, ix);
            const int i = iy * n + ix;
            int rank = 0;
            for (int jy = 0; jy < n; ++jy)
                for (int jx = 0; jx < n; ++jx) {
                    const float vj = val(jy, jx);
                    rank += (vj < vi || (jy * n + jx < i && vj == vi)) ? 1 : 0;
                }
            if (rank == k) {
                r = vi;
                found = true;
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
        // Raster order (the shader's): rows dy, then columns dx.
        for (int dy = 0; dy < n; ++dy) {
            const float* row = s + (threadIdx.y + dy) * TW + threadIdx.x;
            const float* wrow = ws + dy * n;
            for (int dx = 0; dx < n; ++dx) {
                const float nb = row[dx];
                if (nb <= 0.0f) continue;
                const float diff = __fsub_rn(nb, c);
                const float wd = __expf(__fmul_rn(__fmul_rn(-diff, diff), inv_2sd));
                const float wt = __fmul_rn(wrow[dx], wd);
                sum = __fadd_rn(sum, __fmul_rn(nb, wt));
                wsum = __fadd_rn(wsum, wt);
            }
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
