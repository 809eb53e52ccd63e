// CPU restatement of vx-vision's semi-global matching (SGM) stereo path.
//
// TEST INFRASTRUCTURE ONLY: the parity checker for tests/, __graft_entry__.smoke()
// and the CPU-baseline leg of bench.py. Nothing in the product links it.
//
// Parity is pinned: in 2-path mode with subpixel on and no LR check this
// restatement is bit-identical to the reference shader compiled as C++
// (oracle/_ref/libsgm_ref.so) on every golden case in tests/golden/.
#pragma once
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_config {
    int32_t num_disparities;  // 1..256
    float p1, p2;             // used as ushort(p) like the shader
    int32_t census_radius_x, census_radius_y;
    int32_t num_paths;        // 2 (reference: (1,0),(0,1)), 4 or 8
    int32_t subpixel;         // 1: parabola refinement (reference behaviour)
    int32_t lr_check;         // 1: left-right consistency check
    int32_t lr_tolerance;     // pixels
    float invalid_value;      // written where the LR check fails
} oracle_config;

typedef struct oracle_stats {
    uint64_t pixel_steps;    // (pixel, path) recurrence evaluations
    uint64_t wrap_steps;     // of those, steps where some u16 result wrapped
    uint64_t wide_values;    // aggregated L values > 255
} oracle_stats;

// Path k of an n-path run, as a unit step (dx, dy). Order: (1,0), (0,1),
// (-1,0), (0,-1), (1,1), (-1,1), (1,-1), (-1,-1).
void oracle_path_dir(int k, int* dx, int* dy);

// Census transform, vx-vision/shaders/SGMStereo.metal:25-66. Out: one u64 per
// pixel, bits 0..31 = the shader's .x word, bits 32..63 = .y.
int oracle_census(const uint8_t* img, size_t pitch, int w, int h, int rx, int ry, uint64_t* out,
                  int nthreads);

// One aggregation path (dx, dy) over the whole image, SGMStereo.metal:72-173.
// L_out (nullable): W*H*D u16, this path's L_r values (HWD order).
// S_acc (nullable): W*H*D u16, L_r added in (mod 2^16) like the shader's +=.
int oracle_path(const uint64_t* census_l, const uint64_t* census_r, int w, int h, int nd, int p1,
                int p2, int dx, int dy, uint16_t* L_out, uint16_t* S_acc, oracle_stats* stats,
                int nthreads);

// Full pipeline on one pair. disparity (f32, W*H) required; disparity_i16,
// S_out (W*H*D u16) nullable. Returns 0 or -1 on bad arguments.
int oracle_sgm(const uint8_t* left, size_t lpitch, const uint8_t* right, size_t rpitch, int w,
               int h, const oracle_config* cfg, float* disparity, int16_t* disparity_i16,
               uint16_t* S_out, oracle_stats* stats, int nthreads);

// WTA + subpixel + optional LR check on a given cost volume S (W*H*D u16).
int oracle_wta(const uint16_t* S, int w, int h, const oracle_config* cfg, float* disparity,
               int16_t* disparity_i16, int nthreads);

// Depth-map post-filters (vx-vision/shaders/DepthFilter.metal), depth_oracle.cpp.
int oracle_depth_median(const float* in, float* out, int w, int h, int radius);
int oracle_depth_bilateral(const float* in, float* out, int w, int h, int radius, float sigma_s,
                           float sigma_d);

// Sparse ORB stereo matcher (vx-vision/shaders/StereoMatch.metal), stereo_oracle.cpp.
// StereoParams without the counts (StereoMatch.metal:17-26).
typedef struct oracle_stereo_config {
    float max_epipolar, min_disparity, max_disparity;
    uint32_t max_hamming;
    float ratio_thresh, fx, fy, cx, cy, baseline;
} oracle_stereo_config;
// StereoMatchResult as the host reads it (vx-vision/src/types.rs:64-70).
typedef struct oracle_stereo_match_record {
    uint32_t left_idx, right_idx;
    float disparity;
    float point_3d[3];
    float pad;
} oracle_stereo_match_record;
// kpts: n x (x, y, response, level); desc: n x 8 words; out: room for n_left
// records. Returns the number of matches (ascending left index) or -1.
int oracle_stereo_match(const float* left_kpts, uint32_t n_left, const float* right_kpts, uint32_t n_right,
                        const uint32_t* left_desc, const uint32_t* right_desc, const oracle_stereo_config* cfg,
                        oracle_stereo_match_record* out, int nthreads);

#ifdef __cplusplus
}
#endif
