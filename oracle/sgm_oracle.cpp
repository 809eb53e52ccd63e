// CPU restatement of vx-vision's SGM stereo path (MisterEkole/vx-rs).
//
// TEST INFRASTRUCTURE ONLY (parity checker and timed CPU baseline); the product
// never links it. Scalar C++ (no SIMD intrinsics), multithreaded over
// independent scanlines / rows with std::thread.
//
// Reference semantics restated here, with the shader lines they follow:
//  * census        SGMStereo.metal:25-66   strict '<' against the centre,
//                  raster order, centre skipped, clamp-to-edge, bit b -> word b/32.
//  * matching cost SGMStereo.metal:131-142 popcount(L ^ R(x-d)); 64 when x-d < 0.
//  * recurrence    SGMStereo.metal:120-172 evaluated per pixel in increasing d with
//                  ONE array prev[] updated in place: the "d-1" option reads the
//                  value already written for the current pixel, the "d+1" option
//                  the previous pixel's. All results are truncated to u16
//                  (ushort) exactly as the shader stores them, so negative
//                  intermediates wrap mod 2^16.
//  * accumulation  SGMStereo.metal:163-165 S += L (u16, wraps), HWD layout.
//  * WTA           SGMStereo.metal:179-214 first minimum (strict '<', init
//                  0xFFFF), parabola fit when 0 < d < D-1 and |denom| > 1e-6.
// Extensions (not in the reference; the shader only ever runs (1,0) and (0,1),
// sgm.rs:197-200): 4 and 8 paths reuse the same recurrence along (-1,0),
// (0,-1) and the four diagonals, each scanline restarting at the pixel where it
// enters the image; an optional left-right check (right-view WTA over
// S(x'+d, y, d), first minimum over d with x'+d < W; a pixel is invalid when
// x - dL < 0 or |dL - dR(x - dL)| > tolerance).
#include "sgm_oracle.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

namespace {

template <typename F>
void parallel_for(int n, int nthreads, F f) {
    if (n <= 0) return;
    if (nthreads <= 0) nthreads = (int)std::max(1u, std::thread::hardware_concurrency());
    nthreads = std::min(nthreads, n);
    std::atomic<int> next{0};
    auto body = [&]() {
        for (;;) {
            int i = next.fetch_add(1);
            if (i >= n) break;
            f(i);
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nthreads; ++t) pool.emplace_back(body);
    body();
    for (auto& t : pool) t.join();
}

inline int popcount64(uint64_t v) { return __builtin_popcountll(v); }

const int kDirs[8][2] = {{1, 0}, {0, 1}, {-1, 0}, {0, -1}, {1, 1}, {-1, 1}, {1, -1}, {-1, -1}};

// Number of scanlines for direction (dx, dy) and the entry pixel of scanline s.
int num_scanlines(int w, int h, int dx, int dy) {
    if (dy == 0) return h;
    if (dx == 0) return w;
    return w + h - 1;
}

void scanline_start(int w, int h, int dx, int dy, int s, int* x0, int* y0) {
    if (dy == 0) {
        *y0 = s;
        *x0 = dx > 0 ? 0 : w - 1;
    } else if (dx == 0) {
        *x0 = s;
        *y0 = dy > 0 ? 0 : h - 1;
    } else if (s < w) {  // enters through the first row it meets
        *x0 = s;
        *y0 = dy > 0 ? 0 : h - 1;
    } else {  // enters through the first column it meets, below/above that row
        int k = s - w + 1;  // 1..h-1
        *x0 = dx > 0 ? 0 : w - 1;
        *y0 = dy > 0 ? k : h - 1 - k;
    }
}

}  // namespace

extern "C" {

void oracle_path_dir(int k, int* dx, int* dy) {
    *dx = kDirs[k & 7][0];
    *dy = kDirs[k & 7][1];
}

int oracle_census(const uint8_t* img, size_t pitch, int w, int h, int rx, int ry, uint64_t* out,
                  int nthreads) {
    if (!img || !out || w <= 0 || h <= 0 || rx < 0 || ry < 0) return -1;
    if ((2 * rx + 1) * (2 * ry + 1) - 1 > 64) return -1;
    parallel_for(h, nthreads, [&](int y) {
        for (int x = 0; x < w; ++x) {
            const int c = img[(size_t)y * pitch + x];
            uint64_t bits = 0;
            int b = 0;
            for (int dy = -ry; dy <= ry; ++dy) {
                const int sy = std::min(std::max(y + dy, 0), h - 1);
                for (int dx = -rx; dx <= rx; ++dx) {
                    if (dx == 0 && dy == 0) continue;
                    const int sx = std::min(std::max(x + dx, 0), w - 1);
                    if (img[(size_t)sy * pitch + sx] < c) bits |= (uint64_t)1 << b;
                    ++b;
                }
            }
            out[(size_t)y * w + x] = bits;
        }
    });
    return 0;
}

int oracle_path(const uint64_t* cl, const uint64_t* cr, int w, int h, int nd, int p1, int p2,
                int dx, int dy, uint16_t* L_out, uint16_t* S_acc, oracle_stats* stats,
                int nthreads) {
    if (!cl || !cr || w <= 0 || h <= 0 || nd <= 0 || nd > 256) return -1;
    if ((dx == 0 && dy == 0) || dx < -1 || dx > 1 || dy < -1 || dy > 1) return -1;
    const int ns = num_scanlines(w, h, dx, dy);
    std::atomic<uint64_t> steps{0}, wraps{0}, wide{0};
    parallel_for(ns, nthreads, [&](int s) {
        int x, y;
        scanline_start(w, h, dx, dy, s, &x, &y);
        uint16_t prev[256];
        for (int d = 0; d < nd; ++d) prev[d] = 0;
        uint16_t prev_min = 0;
        uint64_t my_steps = 0, my_wraps = 0, my_wide = 0;
        for (int step = 0; x >= 0 && x < w && y >= 0 && y < h; ++step, x += dx, y += dy) {
            const size_t pix = (size_t)y * w + x;
            const uint64_t lc = cl[pix];
            uint16_t cur_min = 0xFFFF;
            bool wrapped = false;
            for (int d = 0; d < nd; ++d) {
                const int xr = x - d;
                const int cost = xr < 0 ? 64 : popcount64(lc ^ cr[(size_t)y * w + xr]);
                uint16_t agg;
                if (step == 0) {
                    agg = (uint16_t)cost;
                } else {
                    // prev[d-1] already holds this pixel's value (in-place update).
                    const int e1 = d > 0 ? prev[d - 1] + p1 : 0xFFFF;
                    const int e2 = d < nd - 1 ? prev[d + 1] + p1 : 0xFFFF;
                    const int e3 = prev_min + p2;
                    const uint16_t o0 = prev[d];
                    const uint16_t o1 = (uint16_t)e1;
                    const uint16_t o2 = (uint16_t)e2;
                    const uint16_t o3 = (uint16_t)e3;
                    const uint16_t best = std::min(std::min(o0, o1), std::min(o2, o3));
                    const int exact = cost + best - prev_min;
                    agg = (uint16_t)exact;
                    if (e1 > 0xFFFF || e2 > 0xFFFF || e3 > 0xFFFF || exact < 0 || exact > 0xFFFF)
                        wrapped = true;
                }
                if (agg > 255) ++my_wide;
                const size_t idx = pix * (size_t)nd + d;
                if (L_out) L_out[idx] = agg;
                if (S_acc) S_acc[idx] = (uint16_t)(S_acc[idx] + agg);
                prev[d] = agg;
                cur_min = std::min(cur_min, agg);
            }
            prev_min = cur_min;
            ++my_steps;
            my_wraps += wrapped;
        }
        steps += my_steps;
        wraps += my_wraps;
        wide += my_wide;
    });
    if (stats) {
        stats->pixel_steps += steps.load();
        stats->wrap_steps += wraps.load();
        stats->wide_values += wide.load();
    }
    return 0;
}

int oracle_wta(const uint16_t* S, int w, int h, const oracle_config* cfg, float* disparity,
               int16_t* disparity_i16, int nthreads) {
    if (!S || !cfg || !disparity || w <= 0 || h <= 0) return -1;
    const int nd = cfg->num_disparities;
    if (nd <= 0 || nd > 256) return -1;
    parallel_for(h, nthreads, [&](int y) {
        std::vector<int> dl(w), dr(w);
        std::vector<float> disp(w);
        for (int x = 0; x < w; ++x) {
            const uint16_t* s = S + ((size_t)y * w + x) * nd;
            uint16_t best_cost = 0xFFFF;
            int best_d = 0;
            for (int d = 0; d < nd; ++d)
                if (s[d] < best_cost) {
                    best_cost = s[d];
                    best_d = d;
                }
            float v = (float)best_d;
            if (cfg->subpixel && best_d > 0 && best_d < nd - 1) {
                const float c0 = (float)s[best_d - 1];
                const float c1 = (float)best_cost;
                const float c2 = (float)s[best_d + 1];
                const float denom = 2.0f * (c0 + c2 - 2.0f * c1);
                if (std::fabs(denom) > 1e-6f) v += (c0 - c2) / denom;
            }
            dl[x] = best_d;
            disp[x] = v;
        }
        if (cfg->lr_check) {
            for (int xr = 0; xr < w; ++xr) {
                uint16_t best_cost = 0xFFFF;
                int best_d = 0;
                for (int d = 0; d < nd && xr + d < w; ++d) {
                    const uint16_t c = S[((size_t)y * w + xr + d) * nd + d];
                    if (c < best_cost) {
                        best_cost = c;
                        best_d = d;
                    }
                }
                dr[xr] = best_d;
            }
        }
        for (int x = 0; x < w; ++x) {
            bool valid = true;
            if (cfg->lr_check) {
                const int xr = x - dl[x];
                valid = xr >= 0 && std::abs(dl[x] - dr[xr]) <= cfg->lr_tolerance;
            }
            disparity[(size_t)y * w + x] = valid ? disp[x] : cfg->invalid_value;
            if (disparity_i16) disparity_i16[(size_t)y * w + x] = (int16_t)(valid ? dl[x] : -1);
        }
    });
    return 0;
}

int oracle_sgm(const uint8_t* left, size_t lpitch, const uint8_t* right, size_t rpitch, int w,
               int h, const oracle_config* cfg, float* disparity, int16_t* disparity_i16,
               uint16_t* S_out, oracle_stats* stats, int nthreads) {
    if (!left || !right || !cfg || !disparity || w <= 0 || h <= 0) return -1;
    const int nd = cfg->num_disparities;
    if (nd <= 0 || nd > 256) return -1;
    if (!(cfg->p1 >= 0.0f && cfg->p1 < 65536.0f && cfg->p2 >= 0.0f && cfg->p2 < 65536.0f))
        return -1;
    const int np = cfg->num_paths;
    if (np != 2 && np != 4 && np != 8) return -1;
    const int p1 = (uint16_t)cfg->p1;  // ushort(params.p1), SGMStereo.metal:155
    const int p2 = (uint16_t)cfg->p2;
    const size_t npx = (size_t)w * h;
    std::vector<uint64_t> cl(npx), cr(npx);
    if (oracle_census(left, lpitch, w, h, cfg->census_radius_x, cfg->census_radius_y, cl.data(),
                      nthreads) != 0)
        return -1;
    if (oracle_census(right, rpitch, w, h, cfg->census_radius_x, cfg->census_radius_y, cr.data(),
                      nthreads) != 0)
        return -1;
    std::vector<uint16_t> S(npx * (size_t)nd, 0);
    for (int k = 0; k < np; ++k) {
        int dx, dy;
        oracle_path_dir(k, &dx, &dy);
        oracle_path(cl.data(), cr.data(), w, h, nd, p1, p2, dx, dy, nullptr, S.data(), stats,
                    nthreads);
    }
    if (oracle_wta(S.data(), w, h, cfg, disparity, disparity_i16, nthreads) != 0) return -1;
    if (S_out) std::memcpy(S_out, S.data(), S.size() * sizeof(uint16_t));
    return 0;
}

}  // extern "C"
