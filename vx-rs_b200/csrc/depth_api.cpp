// DepthFilter entry points of the vx_sgm C ABI (vx-vision/src/kernels/depth_filter.rs).
#include <cmath>

#include "vx_internal.hpp"

using namespace vxsgm;

// The reference's DepthFilter (depth_filter.rs:66-100): compiled pipelines.
// Here: the context the filters run on.
struct vx_depth_filter {
    vx_ctx* ctx = nullptr;
};

namespace {

vx_status check_images(const vx_image* in, const vx_image* out) {
    if (!in || !out) return fail(VX_ERR_INVALID_ARGUMENT, "depth filter: NULL image");
    if (in->format != VX_FORMAT_F32 || out->format != VX_FORMAT_F32)
        return fail(VX_ERR_INVALID_ARGUMENT, "depth filter: images must be F32");
    if (in->width != out->width || in->height != out->height)
        return fail(VX_ERR_SIZE_MISMATCH, "depth filter: input and output sizes differ");
    if (in->ptr == out->ptr) return fail(VX_ERR_INVALID_ARGUMENT, "depth filter: input and output must differ");
    return VX_OK;
}

vx_status finish(vx_ctx* ctx, cudaError_t e, cudaStream_t s, bool sync, const char* what) {
    if (e != cudaSuccess) return cuda_fail(e, what);
    if (sync) {
        e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return cuda_fail(e, what);
    }
    (void)ctx;
    return VX_OK;
}

}  // namespace

extern "C" {

void vx_depth_filter_config_default(vx_depth_filter_config* cfg) {
    if (cfg) *cfg = vx_depth_filter_config{3, 5.0f, 0.05f};  // depth_filter.rs:31-39
}

void vx_depth_median_config_default(vx_depth_median_config* cfg) {
    if (cfg) *cfg = vx_depth_median_config{1};                  // depth_filter.rs:58-62
}

vx_status vx_depth_filter_create(vx_ctx* ctx, vx_depth_filter** out) {
    if (!ctx || !out) return fail(VX_ERR_INVALID_ARGUMENT, "vx_depth_filter_create: NULL argument");
    *out = new vx_depth_filter{ctx};
    return VX_OK;
}

void vx_depth_filter_destroy(vx_depth_filter* f) { delete f; }

vx_status vx_depth_filter_apply_median(vx_depth_filter* f, vx_ctx* ctx, const vx_image* in, vx_image* out,
                                       const vx_depth_median_config* cfg, vx_stream stream) {
    if (!f || !ctx || !cfg) return fail(VX_ERR_INVALID_ARGUMENT, "apply_median: NULL argument");
    vx_status st = check_images(in, out);
    if (st != VX_OK) return st;
    if (cfg->radius < 0 || cfg->radius > kMaxMedianRadius)
        return fail(VX_ERR_INVALID_CONFIG, "apply_median: radius %d not in 0..%d", cfg->radius, kMaxMedianRadius);
    DeviceGuard g(ctx->device);
    cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
    cudaError_t e = launch_depth_median(static_cast<const float*>(in->ptr), in->pitch, static_cast<float*>(out->ptr),
                                        out->pitch, (int)in->width, (int)in->height, cfg->radius, s);
    return finish(ctx, e, s, stream == nullptr, "depth median");
}

vx_status vx_depth_filter_apply_bilateral(vx_depth_filter* f, vx_ctx* ctx, const vx_image* in, vx_image* out,
                                          const vx_depth_filter_config* cfg, vx_stream stream) {
    if (!f || !ctx || !cfg) return fail(VX_ERR_INVALID_ARGUMENT, "apply_bilateral: NULL argument");
    vx_status st = check_images(in, out);
    if (st != VX_OK) return st;
    if (cfg->radius < 0 || cfg->radius > kMaxBilateralRadius)
        return fail(VX_ERR_INVALID_CONFIG, "apply_bilateral: radius %d not in 0..%d", cfg->radius,
                    kMaxBilateralRadius);
    if (!(cfg->sigma_spatial > 0.0f) || !(cfg->sigma_depth > 0.0f) || !std::isfinite(cfg->sigma_spatial) ||
        !std::isfinite(cfg->sigma_depth))
        return fail(VX_ERR_INVALID_CONFIG, "apply_bilateral: sigmas must be finite and > 0");
    DeviceGuard g(ctx->device);
    cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
    cudaError_t e = launch_depth_bilateral(static_cast<const float*>(in->ptr), in->pitch,
                                           static_cast<float*>(out->ptr), out->pitch, (int)in->width,
                                           (int)in->height, cfg->radius, cfg->sigma_spatial, cfg->sigma_depth, s);
    return finish(ctx, e, s, stream == nullptr, "depth bilateral");
}

}  // extern "C"
