// Host-side launchers of the SGM kernels (implemented in the .cu files).
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>

#include "kernels.cuh"

namespace vxsgm {

// Kernel launches issued by this library since load (bench/test evidence).
extern std::atomic<uint64_t> g_kernel_launches;
inline void count_launch(uint64_t n = 1) { g_kernel_launches.fetch_add(n, std::memory_order_relaxed); }
// Device and pinned-host memory allocations this library has requested since
// load (pool allocations, cudaMalloc*, cudaMallocHost), successful or not.
extern std::atomic<uint64_t> g_memory_allocs;
inline void count_alloc() { g_memory_allocs.fetch_add(1, std::memory_order_relaxed); }

// Census of both views of every pair: one CTA per 32x8 tile. banded: also
// write the 32-row banded copy (read only by the single-scanline aggregation).
cudaError_t launch_census(const PairDev* d_pairs, int num_pairs, int total_tiles, int max_rx,
                          int max_ry, bool census64, bool banded, cudaStream_t stream);

// Matching-cost volume of every pair (cost.cu), for batches run by the
// scanline-pair kernel: one CTA per image row of the batch.
cudaError_t prepare_cost_kernels();   // shared-memory limit; once per device
cudaError_t launch_costs(const PairDev* d_pairs, int num_pairs, int total_rows, int dp_max, bool census64,
                         cudaStream_t stream);

// Path aggregation: one persistent launch over the warp units of every (pair,
// path) of a batch. One CTA per SM with `L.warpgroups` warpgroups sharing one
// tensor-memory allocation for the scanline state; warps pull units from the
// plan's queue classes (L.queues, counters[c] per class, zero on entry).
// dp_max / dp_min = largest / smallest padded disparity count of the batch.
// Two forms, picked by the plan's unit size: units of kUnitScanlines (64)
// scanlines run the scanline-pair kernel (aggregate.cu, per-warpgroup TMEM
// budgets and class queues), units of 32 the single-scanline kernel
// (aggregate_single.cu, one queue). wide_tiles: the batch has wide-slab pairs.
// compact: the batch has pairs with a shadow pool (their kernels write the
// escape slot into the byte rows).
struct AggLaunch {
    int warpgroups = 1;
    int tmem_cols = 32;     // scanline-pair kernel: TMEM allocation (power of two >= the budgets' sum)
    AggQueues queues{};
};
cudaError_t prepare_aggregate_kernels();  // shared-memory limits of both; once per device
int aggregate_max_warpgroups(int unit_scanlines, int dp_max, int dp_min, bool census64, bool wide_tiles);
cudaError_t launch_aggregate(int unit_scanlines, int dp_max, int dp_min, bool census64, bool wide_tiles, const AggLaunch& L,
                             const PairDev* d_pairs, const JobDev* d_jobs, const UnitDev* d_units,
                             int num_units, unsigned* counters, cudaStream_t stream, bool compact = false);
namespace pairs {
cudaError_t prepare();
int max_warpgroups(int dp_max, int dp_min, bool wide_tiles);
double budgets_for(const int* dps, const double* work, int n_dps, int warpgroups, int* cols);
// Warpgroups a CTA for a batch of path_pd path-pixel-disparities whose longest
// unit is a chain of chain_steps (pixel step x D) updates.
int default_warpgroups(const int* dps, const double* work, int n_dps, bool wide_tiles, double path_pd,
                       double chain_steps);
cudaError_t launch(int dp_max, bool wide_tiles, const AggLaunch& L, const PairDev* d_pairs,
                   const JobDev* d_jobs, const UnitDev* d_units, int num_units, unsigned* counters,
                   cudaStream_t stream, bool compact = false);
}  // namespace pairs
namespace scan {
cudaError_t launch(const PairDev* d_pairs, const JobDev* d_jobs, const UnitDev* d_units, int num_units,
                   unsigned* counter, cudaStream_t stream, bool compact = false);
}  // namespace scan
namespace single {
cudaError_t prepare();
int max_warpgroups(int dp_max, bool census64);
int default_warpgroups(int dp_max, bool census64, int num_units);
cudaError_t launch(int dp_max, bool census64, int warpgroups, const PairDev* d_pairs, const JobDev* d_jobs,
                   const UnitDev* d_units, int num_units, unsigned* counter, cudaStream_t stream,
                   bool compact = false);
}  // namespace single

// WTA + subpixel + optional LR check: one CTA per (pair, row). The kernel keeps
// three words per pixel of the row in shared memory.
size_t wta_smem_bytes(int max_width);
// Raises the kernel's dynamic shared-memory limit; once per device.
cudaError_t prepare_wta_kernel();
cudaError_t launch_wta(const PairDev* d_pairs, int num_pairs, int total_rows, int max_width,
                       cudaStream_t stream);

// Depth-map post-filters (depth_filter.cu) on pitched F32 planes; radius of the
// median 0..5, of the bilateral 0..kMaxBilateralRadius.
constexpr int kMaxMedianRadius = 5;
constexpr int kMaxBilateralRadius = 32;
cudaError_t launch_depth_median(const float* in, size_t in_pitch, float* out, size_t out_pitch, int W, int H,
                                int radius, cudaStream_t stream);
cudaError_t launch_depth_bilateral(const float* in, size_t in_pitch, float* out, size_t out_pitch, int W, int H,
                                   int radius, float sigma_s, float sigma_d, cudaStream_t stream);

// The depth chain's ends (cloud.cu): RGBA8 -> U8 gray, and the unprojection of
// an F32 depth map to 36-byte GpuPoint3D records (tile_counts: one word per
// depth_to_cloud_tiles() tile; count: the number of pixels that passed).
cudaError_t launch_rgba_to_gray(const uint8_t* in, size_t in_pitch, uint8_t* out, size_t out_pitch, int W, int H,
                                cudaStream_t stream);
int depth_to_cloud_tiles(int W, int H);
cudaError_t launch_depth_to_cloud(const float* depth, size_t depth_pitch, const uint8_t* color, size_t color_pitch,
                                  bool color_rgba, int W, int H, float fx, float fy, float cx, float cy,
                                  float min_depth, float max_depth, float depth_scale, uint32_t max_points,
                                  uint32_t* tile_counts, float* points, uint32_t* count, cudaStream_t stream);

// Sparse ORB stereo matching (stereo_match.cu). Keypoints are CornerPoint
// records read as float4 (x, y, response, level bits); descriptors are 8 words
// per keypoint read as two uint4; both 16-byte aligned. n_right < 2^23.
constexpr uint32_t kStereoMaxRight = (1u << 23) - 1u;
constexpr uint32_t kStereoMaxLeft = 1u << 26;
struct StereoMatchParams {
    uint32_t n_left, n_right;
    float max_epipolar, min_disparity, max_disparity;
    uint32_t max_hamming;  // already cast to 16 bits
    float fx, fy, cx, cy, baseline;
    uint32_t splits, chunk;  // set by launch_stereo_match from the shape
};
// StereoMatchResult as the host reads it (vx-vision/src/types.rs:64-70).
struct StereoMatchRecord {
    uint32_t left_idx, right_idx;
    float disparity;
    float point_3d[3];
    float pad;
};
struct StereoMatchShape {
    uint32_t left_tiles = 0, emit_ctas = 0, splits = 1, chunk = 0;
};
StereoMatchShape stereo_match_shape(uint32_t n_left, uint32_t n_right, int sm_count);
// Scratch: keys (n_left words, all 0xFFFFFFFF between calls), arrivals
// (left_tiles words, all 0 between calls), tile_counts (left_tiles words; the
// banded form's tiles are 32 left keypoints: ceil(n_left / 32) words).
// Both invariants are restored by the launch itself.
cudaError_t launch_stereo_match(const float4* left_kpts, const float4* right_kpts, const uint4* left_desc,
                                const uint4* right_desc, uint32_t* keys, uint32_t* arrivals, uint32_t* tile_counts,
                                StereoMatchRecord* out, uint32_t* count, StereoMatchParams p,
                                const StereoMatchShape& shape, cudaStream_t stream);

// Frames: one launch over n_frames keypoint sets of the concatenated arrays
// (frame f: left [left_offsets[f], left_offsets[f+1]), right likewise); each
// frame's matches go to out + left_offsets[f] in ascending left index, with
// frame-relative indices, and counts[f] receives their number. No scratch.
cudaError_t launch_stereo_match_frames(const float4* left_kpts, const float4* right_kpts, const uint4* left_desc,
                                       const uint4* right_desc, const uint32_t* left_offsets,
                                       const uint32_t* right_offsets, uint32_t n_frames, StereoMatchRecord* out,
                                       uint32_t* counts, StereoMatchParams p, cudaStream_t stream);

// Banded form (large sets, 0 <= max_epipolar < 2^20): right keypoints
// counting-sorted into 1-pixel row buckets 0..kRowBuckets-1 plus one bucket
// for every other y. hist (kRowBuckets + 1) and arrival (1) are 0 between
// calls (restored by the launch); row_start (kRowBuckets + 2) and cursor
// (kRowBuckets + 1) are rewritten by each call; pos/desc/idx hold n_right
// sorted copies (desc: two uint4 per keypoint).
constexpr int kRowBuckets = 8192;
constexpr float kStereoBandMaxEpipolar = 1048576.0f;  // 2^20
struct StereoBandScratch {
    uint32_t* hist = nullptr;
    uint32_t* arrival = nullptr;
    uint32_t* row_start = nullptr;
    uint32_t* cursor = nullptr;
    float2* pos = nullptr;
    uint4* desc = nullptr;
    uint32_t* idx = nullptr;
};
cudaError_t launch_stereo_match_banded(const float4* left_kpts, const float4* right_kpts, const uint4* left_desc,
                                       const uint4* right_desc, const StereoBandScratch& band, uint32_t* keys,
                                       uint32_t* tile_counts, StereoMatchRecord* out, uint32_t* count,
                                       StereoMatchParams p, int sm_count, cudaStream_t stream);

}  // namespace vxsgm
