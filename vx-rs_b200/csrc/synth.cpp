// Seeded synthetic stereo pairs. See synth.h.
//
// Random numbers: SplitMix64 (Steele, Lea & Flood 2014) expands the 64-bit seed
// into the state and stream of a PCG32 generator (O'Neill 2014, XSH-RR output).
// Gaussian samples use the Box-Muller transform. Everything is deterministic
// for a given (scene, w, h, d_lo, d_hi, seed).
#include "synth.h"

#include <algorithm>
#include <cmath>
#include <vector>

namespace {

struct SplitMix64 {
    uint64_t s;
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
};

struct Pcg32 {
    uint64_t state = 0, inc = 1;
    explicit Pcg32(uint64_t seed) {
        SplitMix64 sm{seed};
        inc = (sm.next() << 1) | 1u;
        state = sm.next();
        next();
    }
    uint32_t next() {
        uint64_t old = state;
        state = old * 6364136223846793005ull + inc;
        uint32_t xorshifted = (uint32_t)(((old >> 18u) ^ old) >> 27u);
        uint32_t rot = (uint32_t)(old >> 59u);
        return (xorshifted >> rot) | (xorshifted << ((32u - rot) & 31u));
    }
    double uniform() { return next() * (1.0 / 4294967296.0); }  // [0, 1)
    double uniform(double a, double b) { return a + (b - a) * uniform(); }
    int uniform_int(int a, int b) { return a + (int)(uniform() * (double)(b - a + 1)); }  // [a,b]
    double gauss() {
        double u1 = uniform();
        double u2 = uniform();
        if (u1 < 1e-300) u1 = 1e-300;
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    }
};

// Uniform noise, Gaussian blur (sigma 1.5, radius 5, clamp-to-edge), rescaled to 0..255.
std::vector<float> textured_image(Pcg32& rng, int w, int h) {
    std::vector<float> a((size_t)w * h), b((size_t)w * h);
    for (auto& v : a) v = (float)rng.uniform();
    const int r = 5;
    const double sigma = 1.5;
    float k[2 * r + 1];
    double ks = 0;
    for (int i = -r; i <= r; ++i) ks += (k[i + r] = (float)std::exp(-(i * i) / (2 * sigma * sigma)));
    for (auto& v : k) v = (float)(v / ks);
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            float s = 0;
            for (int i = -r; i <= r; ++i) s += k[i + r] * a[(size_t)y * w + std::clamp(x + i, 0, w - 1)];
            b[(size_t)y * w + x] = s;
        }
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            float s = 0;
            for (int i = -r; i <= r; ++i) s += k[i + r] * b[(size_t)std::clamp(y + i, 0, h - 1) * w + x];
            a[(size_t)y * w + x] = s;
        }
    float lo = *std::min_element(a.begin(), a.end());
    float hi = *std::max_element(a.begin(), a.end());
    float sc = hi > lo ? 255.0f / (hi - lo) : 0.0f;
    for (auto& v : a) v = (v - lo) * sc;
    return a;
}

struct Rect {
    int x0, y0, x1, y1;
};

Rect random_rect(Pcg32& rng, int w, int h) {
    int rw = rng.uniform_int(std::max(1, w / 8), std::max(1, w / 2));
    int rh = rng.uniform_int(std::max(1, h / 8), std::max(1, h / 2));
    int x0 = rng.uniform_int(0, std::max(0, w - rw));
    int y0 = rng.uniform_int(0, std::max(0, h - rh));
    return {x0, y0, x0 + rw, y0 + rh};
}

}  // namespace

extern "C" int vx_synth_pair(int scene, int w, int h, float d_lo, float d_hi, uint64_t seed,
                             uint8_t* left, uint8_t* right, float* gt_disparity) {
    if (w <= 0 || h <= 0 || !left || !right || !(d_hi >= d_lo) || d_lo < 0) return -1;
    if (scene < VX_SYNTH_PLANES || scene > VX_SYNTH_SURFACE) return -1;
    Pcg32 rng(seed);
    const size_t n = (size_t)w * h;
    std::vector<float> L = textured_image(rng, w, h);
    std::vector<float> D(n);
    const int nrect = 8;

    if (scene == VX_SYNTH_SLANTED) {
        // Each region is a plane d = a + gx*(x-cx) + gy*(y-cy) with |(gx,gy)| <= 0.2.
        auto plane = [&](Rect r, bool whole) {
            double ang = rng.uniform(0, 6.283185307179586);
            double mag = rng.uniform(0, 0.2);
            double gx = mag * std::cos(ang), gy = mag * std::sin(ang);
            double a = rng.uniform(d_lo, d_hi);
            double cx = 0.5 * (r.x0 + r.x1), cy = 0.5 * (r.y0 + r.y1);
            int x0 = whole ? 0 : r.x0, x1 = whole ? w : r.x1;
            int y0 = whole ? 0 : r.y0, y1 = whole ? h : r.y1;
            for (int y = y0; y < y1; ++y)
                for (int x = x0; x < x1; ++x)
                    D[(size_t)y * w + x] =
                        (float)std::clamp(a + gx * (x - cx) + gy * (y - cy), (double)d_lo, (double)d_hi);
        };
        plane({0, 0, w, h}, true);
        for (int i = 0; i < nrect; ++i) plane(random_rect(rng, w, h), false);
    } else {
        std::fill(D.begin(), D.end(), (float)rng.uniform_int((int)std::ceil(d_lo), (int)std::floor(d_hi)));
        for (int i = 0; i < nrect; ++i) {
            Rect r = random_rect(rng, w, h);
            float d = (float)rng.uniform_int((int)std::ceil(d_lo), (int)std::floor(d_hi));
            for (int y = r.y0; y < r.y1; ++y)
                for (int x = r.x0; x < r.x1; ++x) D[(size_t)y * w + x] = d;
        }
        if (scene == VX_SYNTH_SURFACE) {
            // Sinusoidal surface over one region, amplitude 20 px around its mean.
            Rect r = random_rect(rng, w, h);
            double base = rng.uniform(std::min((double)d_hi, d_lo + 20.0), std::max((double)d_lo, d_hi - 20.0));
            double lx = rng.uniform(40, 160), ly = rng.uniform(40, 160);
            for (int y = r.y0; y < r.y1; ++y)
                for (int x = r.x0; x < r.x1; ++x)
                    D[(size_t)y * w + x] = (float)std::clamp(
                        base + 20.0 * std::sin(6.283185307179586 * x / lx) * std::sin(6.283185307179586 * y / ly),
                        (double)d_lo, (double)d_hi);
            // Textureless patches covering ~10% of the image: constant +/- N(0,1).
            size_t covered = 0;
            while (covered * 10 < n) {
                int pw = rng.uniform_int(std::max(2, w / 16), std::max(2, w / 6));
                int ph = rng.uniform_int(std::max(2, h / 16), std::max(2, h / 6));
                int x0 = rng.uniform_int(0, std::max(0, w - pw));
                int y0 = rng.uniform_int(0, std::max(0, h - ph));
                float c = (float)rng.uniform(20, 235);
                for (int y = y0; y < std::min(h, y0 + ph); ++y)
                    for (int x = x0; x < std::min(w, x0 + pw); ++x)
                        L[(size_t)y * w + x] = c + (float)rng.gauss();
                covered += (size_t)pw * ph;
            }
        }
    }

    for (size_t i = 0; i < n; ++i) left[i] = (uint8_t)std::clamp(std::lround(L[i]), 0L, 255L);

    // Forward warp with a z-buffer: the larger disparity (nearer surface) wins.
    std::vector<float> zb(n, -1.0f);
    std::vector<float> R(n, 0.0f);
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            const size_t i = (size_t)y * w + x;
            const long xr = std::lround((double)x - D[i]);
            if (xr < 0 || xr >= w) continue;
            const size_t j = (size_t)y * w + xr;
            if (D[i] > zb[j]) {
                zb[j] = D[i];
                R[j] = (float)left[i];
            }
        }
    for (size_t j = 0; j < n; ++j) {
        double v = zb[j] < 0 ? rng.uniform(0, 256) : R[j] + 2.0 * rng.gauss();
        right[j] = (uint8_t)std::clamp(std::lround(v), 0L, 255L);
    }
    if (gt_disparity)
        for (size_t i = 0; i < n; ++i) gt_disparity[i] = D[i];
    return 0;
}
