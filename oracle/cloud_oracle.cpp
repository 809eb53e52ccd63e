// CPU restatement of vx-vision's RGBA -> gray conversion and depth-map
// unprojection ("tier 2" oracle; the reference shaders compiled as C++ are
// tier 1).
//
// TEST INFRASTRUCTURE ONLY: the checker of the CUDA kernels in cloud.cu, never
// part of the product.
//
//  * oracle_rgba_to_gray follows vx-vision/shaders/ColorConvert.metal:21-32:
//    channels read as byte / 255, gray = 0.299 r + 0.587 g + 0.114 b in single
//    precision in that order, written to an 8-bit unorm (clamp to [0, 1], x 255,
//    round to nearest even).
//  * oracle_depth_to_cloud follows vx-vision/shaders/DepthToCloud.metal:30-70
//    with the pixels visited in row-major order (the order in which the
//    shader's atomic counter hands out slots when the pixels run one at a time).
#include <cmath>
#include <cstdint>
#include <cstring>

extern "C" int oracle_rgba_to_gray(const uint8_t* rgba, uint8_t* gray, int w, int h) {
    if (!rgba || !gray || w <= 0 || h <= 0) return -1;
    for (long i = 0; i < (long)w * h; ++i) {
        const float r = (float)rgba[4 * i] / 255.0f, g = (float)rgba[4 * i + 1] / 255.0f,
                    b = (float)rgba[4 * i + 2] / 255.0f;
        float v = 0.299f * r;
        v = v + 0.587f * g;
        v = v + 0.114f * b;
        v = v < 0.0f ? 0.0f : (v > 1.0f ? 1.0f : v);
        gray[i] = (uint8_t)std::nearbyintf(v * 255.0f);
    }
    return 0;
}

// Records of 9 words: x, y, z, 0, colour (r, g, b, a bytes), 0, 0, 0, 0.
// color_format: 0 none, 1 U8, 2 RGBA8 (w x h). Returns the number of pixels
// that passed; writes the first min(that, max_points) records.
extern "C" long oracle_depth_to_cloud(const float* depth, int w, int h, const uint8_t* color, int color_format,
                                      float fx, float fy, float cx, float cy, float min_depth, float max_depth,
                                      float depth_scale, unsigned max_points, void* points) {
    if (!depth || w <= 0 || h <= 0) return -1;
    if (w <= 1) color_format = 0;   // the shader samples colour only from a texture wider than 1 pixel
    unsigned n = 0;
    uint32_t* out = static_cast<uint32_t*>(points);
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            const float d = depth[(long)y * w + x] * depth_scale;
            if (d < min_depth || d > max_depth) continue;   // NaN passes both tests
            const unsigned slot = n++;
            if (slot >= max_points) continue;
            float X = (float)x - cx;
            X = X * d;
            X = X / fx;
            float Y = (float)y - cy;
            Y = Y * d;
            Y = Y / fy;
            uint8_t c[4] = {255, 255, 255, 255};
            if (color_format == 1) c[0] = color[(long)y * w + x], c[1] = 0, c[2] = 0;
            if (color_format == 2) std::memcpy(c, color + 4 * ((long)y * w + x), 3);
            const float zero = 0.0f;
            uint32_t* r = out + 9 * (size_t)slot;
            std::memcpy(r + 0, &X, 4);
            std::memcpy(r + 1, &Y, 4);
            std::memcpy(r + 2, &d, 4);
            std::memcpy(r + 3, &zero, 4);
            std::memcpy(r + 4, c, 4);
            for (int k = 5; k < 9; ++k) std::memcpy(r + k, &zero, 4);
        }
    return (long)n;
}
