// Host driver for the literal reference colour conversion and depth
// unprojection ("tier 1" oracle).
//
// TEST INFRASTRUCTURE ONLY. oracle/Makefile compiles vx-vision's
// shaders/ColorConvert.metal and shaders/DepthToCloud.metal unmodified as C++
// (through oracle/ref_shim) and links them with this file into
// oracle/_ref/libcloud_ref.so. The entry points replay what
// vx-vision/src/kernels/color.rs (ColorConvert::rgba_to_gray) and
// depth_to_cloud.rs (DepthToCloud::compute_raw) encode: one kernel call per
// pixel, here in row-major order, so the shader's atomic point counter hands
// out slots in that order.
#include <cstdint>

#include <metal_stdlib>
using namespace metal;

// Must match vx-vision/shaders/ColorConvert.metal and DepthToCloud.metal field for field.
struct ColorParams {
    uint width;
    uint height;
};
struct GpuPoint3D {
    float px, py, pz;
    float _pad0;
    uchar4 color;
    float nx, ny, nz;
    float _pad1;
};
struct DepthToCloudParams {
    float fx;
    float fy;
    float cx;
    float cy;
    float min_depth;
    float max_depth;
    float depth_scale;
    uint width;
    uint height;
    uint max_points;
};
static_assert(sizeof(GpuPoint3D) == 36, "GpuPoint3D is 36 bytes");

extern "C" void rgba_to_gray(texture2d<float, access::read> input, texture2d<float, access::write> output,
                             const ColorParams& params, uint2 gid);
extern "C" void depth_to_cloud(texture2d<float, access::read> depth_tex, texture2d<float, access::read> color_tex,
                               GpuPoint3D* points, atomic_uint* count, const DepthToCloudParams& params, uint2 gid);

extern "C" int ref_rgba_to_gray(const std::uint8_t* rgba, std::uint8_t* gray, uint width, uint height) {
    texture2d<float, access::read> tin;
    tin.rgba8 = rgba;
    tin.width = tin.pitch = width;
    texture2d<float, access::write> tout;
    tout.u8_out = gray;
    tout.width = tout.pitch = width;
    const ColorParams p{width, height};
    for (uint y = 0; y < height; ++y)
        for (uint x = 0; x < width; ++x) rgba_to_gray(tin, tout, p, uint2(x, y));
    return 0;
}

// color_format: 0 none (the host's 1x1 dummy gray texture), 1 U8 (R8Unorm),
// 2 RGBA8 (RGBA8Unorm), of width x height. points: room for max_points
// records (the host passes min(max_points, W*H)). Returns the counter's value.
extern "C" uint ref_depth_to_cloud(const float* depth, uint width, uint height, const std::uint8_t* color,
                                   int color_format, float fx, float fy, float cx, float cy, float min_depth,
                                   float max_depth, float depth_scale, uint max_points, void* points) {
    texture2d<float, access::read> td;
    td.f32 = const_cast<float*>(depth);
    td.width = td.pitch = width;
    static const std::uint8_t dummy = 0;
    texture2d<float, access::read> tc;
    if (color_format == 2) tc.rgba8 = color;
    else tc.u8 = color_format == 1 ? color : &dummy;
    tc.width = tc.pitch = color_format ? width : 1;
    atomic_uint count{0};
    const DepthToCloudParams p{fx, fy, cx, cy, min_depth, max_depth, depth_scale, width, height, max_points};
    for (uint y = 0; y < height; ++y)
        for (uint x = 0; x < width; ++x)
            depth_to_cloud(td, tc, static_cast<GpuPoint3D*>(points), &count, p, uint2(x, y));
    return count.value;
}
