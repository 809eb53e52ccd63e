// Depth-chain entry points of the vx_sgm C ABI around SGM: RGBA -> gray ingest
// (vx-vision/src/kernels/color.rs, ColorConvert::rgba_to_gray) and depth map ->
// point cloud (vx-vision/src/kernels/depth_to_cloud.rs, DepthToCloud).
#include <algorithm>
#include <cstring>
#include <mutex>

#include "vx_internal.hpp"

using namespace vxsgm;

static_assert(sizeof(vx_point3d) == 36, "GpuPoint3D is 36 bytes (types.rs:440-448)");

// The reference's DepthToCloud (depth_to_cloud.rs:62-64) holds its compiled
// pipeline. Here: the context, the per-tile counts, the device point buffer and
// count of the host-buffer entry point (all grow-only, from the context's pool).
struct vx_depth_to_cloud {
    vx_ctx* ctx = nullptr;
    std::mutex mu;
    uint32_t* tile_counts = nullptr;
    size_t cap_tiles = 0;
    char* dev_points = nullptr;      // count word, then the records
    size_t cap_points = 0;
};

namespace {

vx_status check_color(const vx_image* depth, const vx_image* color) {
    if (!color || color->width <= 1) return VX_OK;   // the reference ignores a color texture of width <= 1
    if (color->format != VX_FORMAT_U8 && color->format != VX_FORMAT_RGBA8)
        return fail(VX_ERR_INVALID_ARGUMENT, "depth_to_cloud: color image must be U8 or RGBA8");
    if (color->width != depth->width || color->height != depth->height)
        return fail(VX_ERR_SIZE_MISMATCH, "depth_to_cloud: color image %ux%u, depth map %ux%u", color->width,
                    color->height, depth->width, depth->height);
    return VX_OK;
}

vx_status ensure_tiles(vx_depth_to_cloud* dc, size_t tiles, cudaStream_t s) {
    if (dc->tile_counts && tiles <= dc->cap_tiles) return VX_OK;
    const size_t cap = std::max(tiles, 2 * dc->cap_tiles);
    if (dc->tile_counts) cudaFreeAsync(dc->tile_counts, s);
    dc->tile_counts = nullptr;
    dc->cap_tiles = 0;
    count_alloc();
    cudaError_t e = cudaMallocFromPoolAsync(reinterpret_cast<void**>(&dc->tile_counts), cap * sizeof(uint32_t),
                                            dc->ctx->pool, s);
    if (e != cudaSuccess) return cuda_fail(e, "depth_to_cloud tile counts");
    dc->cap_tiles = cap;
    return VX_OK;
}

vx_status launch(vx_depth_to_cloud* dc, const vx_image* depth, const vx_image* color, float fx, float fy, float cx,
                 float cy, const vx_depth_to_cloud_config* cfg, uint32_t capacity, vx_point3d* d_points,
                 uint32_t* d_count, cudaStream_t s) {
    const bool use_color = color && color->width > 1;
    vx_status st = ensure_tiles(dc, (size_t)depth_to_cloud_tiles((int)depth->width, (int)depth->height), s);
    if (st != VX_OK) return st;
    cudaError_t e = launch_depth_to_cloud(
        static_cast<const float*>(depth->ptr), depth->pitch, use_color ? static_cast<const uint8_t*>(color->ptr) : nullptr,
        use_color ? color->pitch : 0, use_color && color->format == VX_FORMAT_RGBA8, (int)depth->width,
        (int)depth->height, fx, fy, cx, cy, cfg->min_depth, cfg->max_depth, cfg->depth_scale, capacity,
        dc->tile_counts, reinterpret_cast<float*>(d_points), d_count, s);
    return e == cudaSuccess ? VX_OK : cuda_fail(e, "depth_to_cloud launch");
}

vx_status check_depth(const vx_image* depth, const vx_depth_to_cloud_config* cfg) {
    if (!depth || !cfg) return fail(VX_ERR_INVALID_ARGUMENT, "depth_to_cloud: NULL argument");
    if (depth->format != VX_FORMAT_F32)
        return fail(VX_ERR_INVALID_ARGUMENT, "depth_to_cloud: depth map must be F32 (R32Float)");
    return VX_OK;
}

}  // namespace

extern "C" {

void vx_depth_to_cloud_config_default(vx_depth_to_cloud_config* cfg) {
    if (!cfg) return;
    // DepthToCloudConfig::default(), depth_to_cloud.rs:37-46.
    cfg->min_depth = 0.1f;
    cfg->max_depth = 10.0f;
    cfg->depth_scale = 1.0f;
    cfg->max_points = 1000000u;
}

vx_status vx_depth_to_cloud_create(vx_ctx* ctx, vx_depth_to_cloud** out) {
    if (!ctx || !out) return fail(VX_ERR_INVALID_ARGUMENT, "depth_to_cloud_create: NULL argument");
    auto* dc = new vx_depth_to_cloud;
    dc->ctx = ctx;
    *out = dc;
    return VX_OK;
}

void vx_depth_to_cloud_destroy(vx_depth_to_cloud* dc) {
    if (!dc) return;
    DeviceGuard g(dc->ctx->device);
    if (dc->tile_counts) cudaFreeAsync(dc->tile_counts, dc->ctx->stream);
    if (dc->dev_points) cudaFreeAsync(dc->dev_points, dc->ctx->stream);
    cudaStreamSynchronize(dc->ctx->stream);
    delete dc;
}

vx_status vx_depth_to_cloud_compute_raw(vx_depth_to_cloud* dc, vx_ctx* ctx, const vx_image* depth,
                                        const vx_image* color, float fx, float fy, float cx, float cy,
                                        const vx_depth_to_cloud_config* cfg, vx_point3d* points, size_t capacity,
                                        size_t* n_points) {
    if (!dc || !ctx || !n_points) return fail(VX_ERR_INVALID_ARGUMENT, "depth_to_cloud: NULL argument");
    vx_status st = check_depth(depth, cfg);
    if (st == VX_OK) st = check_color(depth, color);
    if (st != VX_OK) return st;
    // depth_to_cloud.rs:119: at most min(max_points, W*H) points.
    const uint32_t max_pts = (uint32_t)std::min<uint64_t>(cfg->max_points, (uint64_t)depth->width * depth->height);
    if (max_pts > 0 && (!points || capacity < max_pts))
        return fail(VX_ERR_INVALID_ARGUMENT, "depth_to_cloud: capacity %zu < min(max_points, W*H) = %u", capacity,
                    max_pts);
    DeviceGuard g(ctx->device);
    std::lock_guard<std::mutex> lk(dc->mu);
    cudaStream_t s = ctx->stream;
    if (!dc->dev_points || max_pts > dc->cap_points) {
        const size_t cap = std::max<size_t>(max_pts, 2 * dc->cap_points);
        if (dc->dev_points) cudaFreeAsync(dc->dev_points, s);
        dc->dev_points = nullptr;
        dc->cap_points = 0;
        count_alloc();
        cudaError_t e = cudaMallocFromPoolAsync(reinterpret_cast<void**>(&dc->dev_points), 16 + 36 * cap, ctx->pool, s);
        if (e != cudaSuccess) return cuda_fail(e, "depth_to_cloud points");
        dc->cap_points = cap;
    }
    uint32_t* d_count = reinterpret_cast<uint32_t*>(dc->dev_points);
    vx_point3d* d_pts = reinterpret_cast<vx_point3d*>(dc->dev_points + 16);
    st = launch(dc, depth, color, fx, fy, cx, cy, cfg, max_pts, d_pts, d_count, s);
    if (st != VX_OK) return st;
    uint32_t count = 0;
    cudaError_t e = cudaMemcpyAsync(&count, d_count, sizeof count, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    const size_t n = std::min<size_t>(count, max_pts);
    if (e == cudaSuccess && n) e = cudaMemcpyAsync(points, d_pts, n * sizeof(vx_point3d), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(e, "depth_to_cloud");
    *n_points = n;
    return VX_OK;
}

vx_status vx_depth_to_cloud_compute(vx_depth_to_cloud* dc, vx_ctx* ctx, const vx_depth_map* depth,
                                    const vx_image* color, const vx_depth_to_cloud_config* cfg, vx_point3d* points,
                                    size_t capacity, size_t* n_points) {
    if (!depth) return fail(VX_ERR_INVALID_ARGUMENT, "depth_to_cloud: NULL depth map");
    const vx_camera_intrinsics& k = depth->intrinsics;
    return vx_depth_to_cloud_compute_raw(dc, ctx, depth->texture, color, k.fx, k.fy, k.cx, k.cy, cfg, points,
                                         capacity, n_points);
}

vx_status vx_depth_to_cloud_compute_device(vx_depth_to_cloud* dc, vx_ctx* ctx, const vx_image* depth,
                                           const vx_image* color, float fx, float fy, float cx, float cy,
                                           const vx_depth_to_cloud_config* cfg, vx_point3d* d_points,
                                           uint32_t capacity, uint32_t* d_count, vx_stream stream) {
    if (!dc || !ctx || !d_count || (capacity && !d_points))
        return fail(VX_ERR_INVALID_ARGUMENT, "depth_to_cloud_device: NULL argument");
    if (reinterpret_cast<uintptr_t>(d_points) % 4 != 0 || reinterpret_cast<uintptr_t>(d_count) % 4 != 0)
        return fail(VX_ERR_INVALID_ARGUMENT, "depth_to_cloud_device: misaligned buffers");
    vx_status st = check_depth(depth, cfg);
    if (st == VX_OK) st = check_color(depth, color);
    if (st != VX_OK) return st;
    const uint32_t max_pts = (uint32_t)std::min<uint64_t>(
        {(uint64_t)cfg->max_points, (uint64_t)depth->width * depth->height, (uint64_t)capacity});
    DeviceGuard g(ctx->device);
    std::lock_guard<std::mutex> lk(dc->mu);
    cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
    st = launch(dc, depth, color, fx, fy, cx, cy, cfg, max_pts, d_points, d_count, s);
    if (st == VX_OK && !stream) {
        cudaError_t e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) st = cuda_fail(e, "depth_to_cloud");
    }
    return st;
}

vx_status vx_color_rgba_to_gray(vx_ctx* ctx, const vx_image* in, vx_image* out, vx_stream stream) {
    if (!ctx || !in || !out) return fail(VX_ERR_INVALID_ARGUMENT, "rgba_to_gray: NULL argument");
    if (in->format != VX_FORMAT_RGBA8 || out->format != VX_FORMAT_U8)
        return fail(VX_ERR_INVALID_ARGUMENT, "rgba_to_gray: input must be RGBA8 and output U8");
    if (in->width != out->width || in->height != out->height)
        return fail(VX_ERR_SIZE_MISMATCH, "rgba_to_gray: %ux%u into %ux%u", in->width, in->height, out->width,
                    out->height);
    DeviceGuard g(ctx->device);
    cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
    cudaError_t e = launch_rgba_to_gray(static_cast<const uint8_t*>(in->ptr), in->pitch, static_cast<uint8_t*>(out->ptr),
                                        out->pitch, (int)in->width, (int)in->height, s);
    if (e == cudaSuccess && !stream) e = cudaStreamSynchronize(s);
    return e == cudaSuccess ? VX_OK : cuda_fail(e, "rgba_to_gray");
}

}  // extern "C"
