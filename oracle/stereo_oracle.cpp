// CPU restatement of vx-vision's sparse ORB stereo matcher (StereoMatcher):
// shaders/StereoMatch.metal (stereo_hamming + stereo_extract) as driven by
// src/kernels/stereomatch.rs:115-249.
//
// TEST INFRASTRUCTURE ONLY: the parity checker for tests/ and the CPU baseline
// of bench.py. Nothing in the product links it. Parity is pinned: it equals the
// reference shader compiled as C++ (oracle/_ref/libstereo_ref.so) record for
// record on every case of tests/golden/stereo_match_cases.npz.
//
// Restated without the n_left x n_right distance matrix: a left keypoint's row
// of that matrix is consumed as it is produced, which the first-minimum scan of
// stereo_extract allows (it reads the row in ascending right index).
// Scalar C++, std::thread over left keypoints; matches come out in ascending
// left index (the reference appends them through an atomic counter, so its
// order is unspecified; the set of records is the same).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <functional>
#include <thread>
#include <vector>

#include "sgm_oracle.h"

namespace {

// CornerPoint (vx-vision/src/types.rs:8-12).
struct Kpt {
    float x, y, response;
    uint32_t level;
};

// Runs f(begin, end) over [0, n) in blocks of `block` on nthreads threads.
void for_each_block(int64_t n, int nthreads, int64_t block, const std::function<void(int64_t, int64_t)>& f) {
    if (n <= 0) return;
    if (nthreads <= 0) nthreads = (int)std::max(1u, std::thread::hardware_concurrency());
    const int64_t nblocks = (n + block - 1) / block;
    nthreads = (int)std::min<int64_t>(nthreads, nblocks);
    std::atomic<int64_t> next{0};
    auto body = [&]() {
        for (;;) {
            const int64_t b = next.fetch_add(1);
            if (b >= nblocks) break;
            f(b * block, std::min(n, (b + 1) * block));
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nthreads; ++t) pool.emplace_back(body);
    body();
    for (auto& t : pool) t.join();
}

}  // namespace

extern "C" {

// StereoMatch.metal:32-63 (one distance per pair: 0xFFFF unless the epipolar
// test |yl - yr| <= max_epipolar and min_disparity <= xl - xr <= max_disparity
// pass) and :68-115 (first minimum over the row with strict <, reject when it
// exceeds max_hamming cast to ushort, triangulate in the shader's operation
// order). Records: left_idx, right_idx, disparity, X, Y, Z, pad (0).
int oracle_stereo_match(const float* left_kpts, uint32_t n_left, const float* right_kpts, uint32_t n_right,
                        const uint32_t* left_desc, const uint32_t* right_desc, const oracle_stereo_config* cfg,
                        oracle_stereo_match_record* out, int nthreads) {
    if (!cfg || !out) return -1;
    if (n_left == 0 || n_right == 0) return 0;  // stereomatch.rs:138-142
    const Kpt* lk = reinterpret_cast<const Kpt*>(left_kpts);
    const Kpt* rk = reinterpret_cast<const Kpt*>(right_kpts);
    const uint16_t max_ham = static_cast<uint16_t>(cfg->max_hamming);  // ushort(params.max_hamming), :96
    std::vector<uint32_t> best_of(n_left);
    for_each_block(n_left, nthreads, 16, [&](int64_t i0, int64_t i1) {
        for (int64_t i = i0; i < i1; ++i) {
            const Kpt& l = lk[i];
            const uint32_t* ld = left_desc + 8 * i;
            uint16_t best = 0xFFFF;
            uint32_t best_ri = 0;
            for (uint32_t j = 0; j < n_right; ++j) {
                const Kpt& r = rk[j];
                uint16_t dist = 0xFFFF;
                const float dy = std::fabs(l.y - r.y);
                if (dy <= cfg->max_epipolar) {
                    const float d = l.x - r.x;
                    if (d >= cfg->min_disparity && d <= cfg->max_disparity) {
                        const uint32_t* rd = right_desc + 8ull * j;
                        uint32_t s = 0;
                        for (int w = 0; w < 8; ++w) s += (uint32_t)__builtin_popcount(ld[w] ^ rd[w]);
                        dist = static_cast<uint16_t>(s);
                    }
                }
                if (dist < best) {  // the shader's `second` feeds only a disabled ratio test
                    best = dist;
                    best_ri = j;
                }
            }
            best_of[i] = best > max_ham ? 0xFFFFFFFFu : best_ri;
        }
    });
    int n = 0;
    for (uint32_t i = 0; i < n_left; ++i) {
        if (best_of[i] == 0xFFFFFFFFu) continue;
        const uint32_t j = best_of[i];
        const float disp = lk[i].x - rk[j].x;
        const float Z = cfg->fx * cfg->baseline / disp;
        const float X = Z * (lk[i].x - cfg->cx) / cfg->fx;
        const float Y = Z * (lk[i].y - cfg->cy) / cfg->fy;
        out[n] = oracle_stereo_match_record{i, j, disp, {X, Y, Z}, 0.0f};
        ++n;
    }
    return n;
}

}  // extern "C"
