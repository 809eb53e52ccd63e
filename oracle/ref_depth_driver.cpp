// Host driver for the literal reference depth filters ("tier 1" oracle).
//
// TEST INFRASTRUCTURE ONLY. oracle/Makefile compiles vx-vision's
// shaders/DepthFilter.metal unmodified as C++ (through oracle/ref_shim) and links
// it with this file into oracle/_ref/libdepth_ref.so. The entry points replay
// what vx-vision/src/kernels/depth_filter.rs (DepthFilter::apply_bilateral,
// ::apply_median) encodes: one kernel call per pixel of the output.
#include <cstdint>

#include <metal_stdlib>
using namespace metal;

// Must match vx-vision/shaders/DepthFilter.metal field for field.
struct DepthBilateralParams {
    uint width;
    uint height;
    int radius;
    float sigma_spatial;
    float sigma_depth;
};
struct DepthMedianParams {
    uint width;
    uint height;
    int radius;
};

extern "C" void depth_bilateral(texture2d<float, access::read> depth_in,
                                texture2d<float, access::write> depth_out,
                                const DepthBilateralParams& params, uint2 gid);
extern "C" void depth_median(texture2d<float, access::read> depth_in,
                             texture2d<float, access::write> depth_out,
                             const DepthMedianParams& params, uint2 gid);

extern "C" int ref_depth_bilateral(const float* in, float* out, uint width, uint height, int radius,
                                   float sigma_spatial, float sigma_depth) {
    texture2d<float, access::read> tin;
    tin.f32 = const_cast<float*>(in);
    tin.width = tin.pitch = width;
    texture2d<float, access::write> tout;
    tout.f32 = out;
    tout.width = tout.pitch = width;
    const DepthBilateralParams p{width, height, radius, sigma_spatial, sigma_depth};
    for (uint y = 0; y < height; ++y)
        for (uint x = 0; x < width; ++x) depth_bilateral(tin, tout, p, uint2(x, y));
    return 0;
}

extern "C" int ref_depth_median(const float* in, float* out, uint width, uint height, int radius) {
    texture2d<float, access::read> tin;
    tin.f32 = const_cast<float*>(in);
    tin.width = tin.pitch = width;
    texture2d<float, access::write> tout;
    tout.f32 = out;
    tout.width = tout.pitch = width;
    const DepthMedianParams p{width, height, radius};
    for (uint y = 0; y < height; ++y)
        for (uint x = 0; x < width; ++x) depth_median(tin, tout, p, uint2(x, y));
    return 0;
}
