// CPU restatement of vx-vision's depth-map post-filters (DepthFilter): the
// median and the bilateral filter of shaders/DepthFilter.metal.
//
// TEST INFRASTRUCTURE ONLY: the parity checker for tests/. Nothing in the
// product links it. Parity is pinned: it is bit-identical to the reference
// shader compiled as C++ (oracle/_ref/libdepth_ref.so) on every case of
// tests/golden/depth_filter_cases.npz (same float operations in the same order,
// same host expf).
#include <algorithm>
#include <cmath>
#include <vector>

#include "sgm_oracle.h"

namespace {

inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

}  // namespace

extern "C" {

// DepthFilter.metal:84-120 (depth_median): the valid (> 0) values of the
// clamped (2r+1)^2 window in raster order, at most 121 of them; the output is
// the element at index count/2 of their ascending order, or 0 if none is valid.
int oracle_depth_median(const float* in, float* out, int w, int h, int radius) {
    if (!in || !out || w <= 0 || h <= 0) return -1;
    std::vector<float> vals;
    vals.reserve(121);
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            vals.clear();
            for (int dy = -radius; dy <= radius; ++dy)
                for (int dx = -radius; dx <= radius; ++dx) {
                    const float d = in[(size_t)clampi(y + dy, 0, h - 1) * w + clampi(x + dx, 0, w - 1)];
                    if (d > 0.0f && vals.size() < 121) vals.push_back(d);
                }
            float r = 0.0f;
            if (!vals.empty()) {
                const size_t k = vals.size() / 2;
                std::nth_element(vals.begin(), vals.begin() + k, vals.end());
                r = vals[k];
            }
            out[(size_t)y * w + x] = r;
        }
    return 0;
}

// DepthFilter.metal:20-66 (depth_bilateral): for a valid centre, the weighted
// mean of the valid neighbours of the clamped window, weight =
// exp(-(dx^2+dy^2)/(2 ss^2)) * exp(-(n-c)^2/(2 sd^2)); the centre itself when
// the weights sum to at most 1e-8; 0 for a centre <= 0. Single-precision
// arithmetic in the shader's order.
int oracle_depth_bilateral(const float* in, float* out, int w, int h, int radius, float sigma_s,
                           float sigma_d) {
    if (!in || !out || w <= 0 || h <= 0) return -1;
    const float inv_2ss = 1.0f / (2.0f * sigma_s * sigma_s);
    const float inv_2sd = 1.0f / (2.0f * sigma_d * sigma_d);
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            const float c = in[(size_t)y * w + x];
            if (c <= 0.0f) {            // (a NaN centre goes on, as in the shader)
                out[(size_t)y * w + x] = 0.0f;
                continue;
            }
            float sum = 0.0f, wsum = 0.0f;
            for (int dy = -radius; dy <= radius; ++dy)
                for (int dx = -radius; dx <= radius; ++dx) {
                    const float n = in[(size_t)clampi(y + dy, 0, h - 1) * w + clampi(x + dx, 0, w - 1)];
                    if (n <= 0.0f) continue;
                    const float sd2 = (float)(dx * dx + dy * dy);
                    const float ws = std::exp(-sd2 * inv_2ss);
                    const float diff = n - c;
                    const float wd = std::exp(-diff * diff * inv_2sd);
                    const float wt = ws * wd;
                    sum += n * wt;
                    wsum += wt;
                }
            out[(size_t)y * w + x] = wsum > 1e-8f ? sum / wsum : c;
        }
    return 0;
}

}  // extern "C"
