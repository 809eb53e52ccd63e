// Host driver for the literal reference sparse stereo matcher ("tier 1" oracle).
//
// TEST INFRASTRUCTURE ONLY. oracle/Makefile compiles vx-vision's
// shaders/StereoMatch.metal unmodified as C++ (through oracle/ref_shim) and links
// it with this file into oracle/_ref/libstereo_ref.so. ref_stereo_match replays
// what vx-vision/src/kernels/stereomatch.rs:115-249 (StereoMatcher::run) encodes:
// stereo_hamming over the whole n_left x n_right grid into a u16 distance matrix,
// then stereo_extract once per left keypoint. Threads run one at a time in index
// order, so the atomic append yields the matches in ascending left index.
#include <cstdint>
#include <cstring>
#include <vector>

#include <metal_stdlib>
using namespace metal;

// Must match vx-vision/shaders/StereoMatch.metal:4-26 field for field.
struct CornerPoint {
    float2 position;
    float response;
    uint pyramid_level;
};
struct StereoMatchResult {
    uint left_idx;
    uint right_idx;
    float disparity;
    float3 point_3d;
};
struct StereoParams {
    uint n_left;
    uint n_right;
    float max_epipolar;
    float min_disparity;
    float max_disparity;
    uint max_hamming;
    float ratio_thresh;
    float fx, fy, cx, cy, baseline;
};

extern "C" void stereo_hamming(uint32_t* left_desc, uint32_t* right_desc, CornerPoint* left_kpts,
                               CornerPoint* right_kpts, ushort* dist_matrix, const StereoParams& params,
                               uint2 gid);
extern "C" void stereo_extract(ushort* dist_matrix, CornerPoint* left_kpts, CornerPoint* right_kpts,
                               StereoMatchResult* matches, atomic_uint* match_count,
                               const StereoParams& params, uint tid);

// The host-side record (vx-vision/src/types.rs:64-70): 7 four-byte fields.
struct HostMatch {
    uint32_t left_idx, right_idx;
    float disparity;
    float point_3d[3];
    float pad;
};

// kpts: n x 4 floats (x, y, response, level bits); desc: n x 8 words.
// out: room for n_left records. Returns the number of matches.
extern "C" int ref_stereo_match(const float* left_kpts, uint32_t n_left, const float* right_kpts,
                                uint32_t n_right, const uint32_t* left_desc, const uint32_t* right_desc,
                                float max_epipolar, float min_disparity, float max_disparity,
                                uint32_t max_hamming, float ratio_thresh, float fx, float fy, float cx,
                                float cy, float baseline, HostMatch* out) {
    if (n_left == 0 || n_right == 0) return 0;  // stereomatch.rs:138-142
    std::vector<CornerPoint> lk(n_left), rk(n_right);
    std::memcpy(lk.data(), left_kpts, sizeof(CornerPoint) * n_left);
    std::memcpy(rk.data(), right_kpts, sizeof(CornerPoint) * n_right);
    std::vector<uint32_t> ld(left_desc, left_desc + 8ull * n_left), rd(right_desc, right_desc + 8ull * n_right);
    std::vector<ushort> dist(static_cast<size_t>(n_left) * n_right);
    std::vector<StereoMatchResult> matches(n_left);
    atomic_uint count{0};
    const StereoParams p{n_left, n_right, max_epipolar, min_disparity, max_disparity, max_hamming,
                         ratio_thresh, fx, fy, cx, cy, baseline};
    for (uint ri = 0; ri < n_right; ++ri)
        for (uint li = 0; li < n_left; ++li)
            stereo_hamming(ld.data(), rd.data(), lk.data(), rk.data(), dist.data(), p, uint2(li, ri));
    for (uint t = 0; t < n_left; ++t)
        stereo_extract(dist.data(), lk.data(), rk.data(), matches.data(), &count, p, t);
    const uint n = count.value < n_left ? count.value : n_left;  // stereomatch.rs:245
    for (uint i = 0; i < n; ++i) {
        out[i].left_idx = matches[i].left_idx;
        out[i].right_idx = matches[i].right_idx;
        out[i].disparity = matches[i].disparity;
        out[i].point_3d[0] = matches[i].point_3d.x;
        out[i].point_3d[1] = matches[i].point_3d.y;
        out[i].point_3d[2] = matches[i].point_3d.z;
        out[i].pad = 0.0f;
    }
    return static_cast<int>(n);
}
