// Census transform for a batch of stereo pairs (both views in one launch).
//
// Semantics: vx-vision/shaders/SGMStereo.metal:25-66 - bit b of the descriptor
// is set iff neighbour < centre (strict), neighbours in raster order with the
// centre skipped, coordinates clamped to the image. The shader reads R8Unorm
// texels as value/255 floats; comparing those is the same as comparing the
// u8 values, which is what this kernel does.
//
// Layout: each 32x32 tile of one view is staged once in shared memory with its
// (rx, ry) apron, then every thread builds four
// descriptors (rows 8 apart) from shared memory: large tiles, so that the
// per-CTA costs (finding the pair, staging latency) are paid per 1024 pixels. Descriptors are written row-major (read by
// the cost-volume kernel and by the vertical and diagonal paths of the
// single-scanline aggregation) and, for batches run by the single-scanline
// aggregation only, a second time in 32-row bands, x-major inside a band, word
// (x, y) at ((y/32)*W + x)*32 + y%32 (read by its horizontal paths: the 32
// scanlines of a warp are the 32 rows of a band, so each column is 128
// contiguous bytes). Output word: u32 when the window has <= 32 bits, else u64.
//
// Staging. A tile whose apron lies inside the image, of a view whose base and
// pitch are 16-byte aligned, is copied with asynchronous 16-byte copies
// (cp.async, global -> shared without registers): each staged row is the
// 16-byte aligned segment [bx - rx - lead, +rw) with lead = (-rx) mod 16 (bx is
// a multiple of 32), rw = lead + 32 + 2 rx rounded up to 16, read only inside
// the row. Border tiles (and unaligned views) stage byte by byte with clamped
// coordinates, which reproduces the shader's clamp.
#include <cuda_runtime.h>

#include "kernels.cuh"
#include "launch.hpp"

namespace vxsgm {

namespace {

__device__ __forceinline__ int find_pair_by_tile(const PairDev* pairs, int n, int tile) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (pairs[mid].census_tile_begin <= tile) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// Descriptor of the window centred at (cx, cy) of the staged tile (row stride
// sw); RX, RY < 0: the radii rx, ry at run time.
template <int RX, int RY>
__device__ __forceinline__ uint64_t window_bits(const uint8_t* __restrict__ tile_px, int sw, int cx, int cy, int rx,
                                                int ry) {
    if (RX >= 0) {
        rx = RX;
        ry = RY;
    }
    const int c = tile_px[cy * sw + cx];
    uint64_t bits = 0;
    int b = 0;
#pragma unroll
    for (int dy = -ry; dy <= ry; ++dy) {
        const uint8_t* row = tile_px + (cy + dy) * sw + cx;
#pragma unroll
        for (int dx = -rx; dx <= rx; ++dx) {
            if (dx == 0 && dy == 0) continue;
            bits |= (uint64_t)(row[dx] < c) << b;
            ++b;
        }
    }
    return bits;
}

template <typename CT, bool BANDED>
__global__ void __launch_bounds__(kCensusTileW * kCensusThreadsY)
census_kernel(const PairDev* __restrict__ pairs, int num_pairs) {
    extern __shared__ __align__(16) uint8_t tile_px[];
    __shared__ CT tile_bits[kCensusTileH][kCensusTileW + 1];
    constexpr int kRowsPerThread = kCensusTileH / kCensusThreadsY;
    const int pi = find_pair_by_tile(pairs, num_pairs, blockIdx.x);
    const PairDev& pr = pairs[pi];
    const int W = pr.width, H = pr.height, rx = pr.rx, ry = pr.ry;
    const int tiles_x = (W + kCensusTileW - 1) / kCensusTileW;
    const int tiles_y = (H + kCensusTileH - 1) / kCensusTileH;
    int t = blockIdx.x - pr.census_tile_begin;
    const int view = t / (tiles_x * tiles_y);  // 0 = left, 1 = right
    t -= view * tiles_x * tiles_y;
    const int bx = (t % tiles_x) * kCensusTileW;
    const int by = (t / tiles_x) * kCensusTileH;
    const uint8_t* img = view ? pr.right : pr.left;
    const size_t pitch = view ? pr.right_pitch : pr.left_pitch;

    const int sw = kCensusTileW + 2 * rx, sh = kCensusTileH + 2 * ry;
    const int tid = threadIdx.y * kCensusTileW + threadIdx.x;
    constexpr int kThreads = kCensusTileW * kCensusThreadsY;
    const int lead = census_stage_lead(rx), rw = census_stage_row_bytes(rx);
    const int x0 = bx - rx - lead;
    const bool async_stage = ((reinterpret_cast<uintptr_t>(img) | (uintptr_t)pitch) & 15) == 0 && x0 >= 0 &&
                             x0 + rw <= W && by - ry >= 0 && by + kCensusTileH + ry <= H;
    int stride = sw, col0 = 0;           // staged row stride, column of x = bx - rx
    if (async_stage) {
        stride = rw;
        col0 = lead;
        const uint8_t* src = img + (size_t)(by - ry) * pitch + x0;
        const int cpr = rw >> 4;         // 16-byte copies a row
        const uint32_t dst0 = (uint32_t)__cvta_generic_to_shared(tile_px);
        for (int i = tid; i < sh * cpr; i += kThreads) {
            const int r = i / cpr, c = i - r * cpr;
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst0 + (uint32_t)(r * rw + 16 * c)),
                         "l"(src + (size_t)r * pitch + 16 * c)
                         : "memory");
        }
        asm volatile("cp.async.wait_all;" ::: "memory");
    } else {
        for (int i = tid; i < sw * sh; i += kThreads) {
            const int sx = min(max(bx - rx + i % sw, 0), W - 1);
            const int sy = min(max(by - ry + i / sw, 0), H - 1);
            tile_px[i] = img[(size_t)sy * pitch + sx];
        }
    }
    __syncthreads();

    // Clamped reads at the image border equal reads of the staged apron, which
    // was filled with clamped coordinates; interior threads read their window.
    // The common windows (5x5, 9x7) are unrolled; the radii are uniform per CTA.
    CT* rm = static_cast<CT*>(view ? pr.census_r : pr.census_l);
    const int x = bx + threadIdx.x, cx = col0 + threadIdx.x + rx;
#pragma unroll
    for (int k = 0; k < kRowsPerThread; ++k) {
        const int ty = threadIdx.y + k * kCensusThreadsY;
        const int y = by + ty, cy = ty + ry;
        uint64_t bits;
        if (rx == 2 && ry == 2) bits = window_bits<2, 2>(tile_px, stride, cx, cy, rx, ry);
        else if (rx == 4 && ry == 3) bits = window_bits<4, 3>(tile_px, stride, cx, cy, rx, ry);
        else bits = window_bits<-1, -1>(tile_px, stride, cx, cy, rx, ry);
        if (x < W && y < H) rm[(size_t)y * W + x] = (CT)bits;
        if constexpr (BANDED) tile_bits[ty][threadIdx.x] = (CT)bits;
    }
    if constexpr (!BANDED) return;   // the scanline-pair and scan aggregations read the cost volume instead
    // Banded copy: the tile is one 32-row band (by is a multiple of 32), so a
    // tile column is 32 consecutive words there; the descriptors go through
    // shared memory and consecutive threads write consecutive words.
    CT* cm = static_cast<CT*>(view ? pr.census_rt : pr.census_lt);
    __syncthreads();
    for (int w = tid; w < kCensusTileW * kCensusTileH; w += kThreads) {
        const int col = w / kCensusTileH, row = w % kCensusTileH;
        const int ox = bx + col, oy = by + row;
        if (ox < W && oy < H) cm[((size_t)(oy >> 5) * W + ox) * 32 + (oy & 31)] = tile_bits[row][col];
    }
}

}  // namespace

cudaError_t launch_census(const PairDev* d_pairs, int num_pairs, int total_tiles, int max_rx,
                          int max_ry, bool census64, bool banded, cudaStream_t stream) {
    if (total_tiles == 0) return cudaSuccess;
    const dim3 block(kCensusTileW, kCensusThreadsY);
    const size_t smem = census_smem_bytes(max_rx, max_ry);
    count_launch();
    if (census64) {
        if (banded) census_kernel<uint64_t, true><<<total_tiles, block, smem, stream>>>(d_pairs, num_pairs);
        else census_kernel<uint64_t, false><<<total_tiles, block, smem, stream>>>(d_pairs, num_pairs);
    } else {
        if (banded) census_kernel<uint32_t, true><<<total_tiles, block, smem, stream>>>(d_pairs, num_pairs);
        else census_kernel<uint32_t, false><<<total_tiles, block, smem, stream>>>(d_pairs, num_pairs);
    }
    return cudaGetLastError();
}

}  // namespace vxsgm
