// Context, images and error reporting of the vx_sgm C ABI.
#include <cstdio>
#include <algorithm>
#include <cstring>

#include "vx_internal.hpp"

namespace vxsgm {

std::atomic<uint64_t> g_kernel_launches{0};
std::atomic<uint64_t> g_memory_allocs{0};

namespace {
thread_local std::string t_last_error;
}

vx_status fail(vx_status status, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    t_last_error = buf;
    return status;
}

vx_status cuda_fail(cudaError_t err, const char* what) {
    if (err == cudaErrorMemoryAllocation)
        return fail(VX_ERR_BUFFER_ALLOC, "%s: %s", what, cudaGetErrorString(err));
    if (err == cudaErrorNoKernelImageForDevice || err == cudaErrorInvalidKernelImage)
        return fail(VX_ERR_SHADER_MISSING, "%s: %s", what, cudaGetErrorString(err));
    return fail(VX_ERR_GPU, "%s: %s", what, cudaGetErrorString(err));
}

size_t format_bytes(vx_format f) {
    switch (f) {
        case VX_FORMAT_U8: return 1;
        case VX_FORMAT_F32: return 4;
        case VX_FORMAT_I16: return 2;
        case VX_FORMAT_RGBA8: return 4;
    }
    return 0;
}

}  // namespace vxsgm

using namespace vxsgm;

extern "C" {

const char* vx_last_error(void) { return t_last_error.c_str(); }

uint64_t vx_kernel_launch_count(void) { return g_kernel_launches.load(); }

uint64_t vx_memory_allocation_count(void) { return g_memory_allocs.load(); }

vx_status vx_ctx_create(int device_ordinal, vx_ctx** out) {
    if (!out) return fail(VX_ERR_INVALID_ARGUMENT, "vx_ctx_create: out is NULL");
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return fail(VX_ERR_DEVICE_NOT_FOUND, "no CUDA device found");
    }
    if (device_ordinal < 0 || device_ordinal >= count)
        return fail(VX_ERR_DEVICE_NOT_FOUND, "device %d out of range (%d devices)", device_ordinal,
                    count);
    DeviceGuard g(device_ordinal);
    auto* ctx = new vx_ctx;
    ctx->device = device_ordinal;
    cudaError_t e = cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device_ordinal);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) {
        size_t free_b = 0, total_b = 0;
        e = cudaMemGetInfo(&free_b, &total_b);
        ctx->workspace_limit = free_b / 20 * 17;
    }
    if (e == cudaSuccess) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device_ordinal;
        e = cudaMemPoolCreate(&ctx->pool, &props);
    }
    if (e == cudaSuccess) {
        uint64_t threshold = UINT64_MAX;
        e = cudaMemPoolSetAttribute(ctx->pool, cudaMemPoolAttrReleaseThreshold, &threshold);
    }

    if (e != cudaSuccess) {
        vx_status s = cuda_fail(e, "vx_ctx_create");
        if (ctx->pool) cudaMemPoolDestroy(ctx->pool);
        if (ctx->stream) cudaStreamDestroy(ctx->stream);
        delete ctx;
        return s;
    }
    *out = ctx;
    return VX_OK;
}

void vx_ctx_destroy(vx_ctx* ctx) {
    if (!ctx) return;
    DeviceGuard g(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    for (auto ev : ctx->stage_ev) cudaEventDestroy(ev);
    cudaStreamDestroy(ctx->stream);
    cudaMemPoolDestroy(ctx->pool);
    delete ctx;
}

vx_status vx_ctx_enable_stage_timing(vx_ctx* ctx, int enable) {
    if (!ctx) return fail(VX_ERR_INVALID_ARGUMENT, "vx_ctx_enable_stage_timing: ctx is NULL");
    DeviceGuard g(ctx->device);
    std::lock_guard<std::mutex> lk(ctx->timing_mu);
    if (enable && ctx->stage_ev.empty()) {
        ctx->stage_ev.resize(vx_ctx::kTimingSlots * vx_ctx::kStageEvents);
        for (auto& ev : ctx->stage_ev) {
            cudaError_t e = cudaEventCreate(&ev);
            if (e != cudaSuccess) return cuda_fail(e, "creating timing events");
        }
    }
    ctx->timing = enable != 0;
    ctx->timing_batches = 0;
    return VX_OK;
}

cudaEvent_t* vx_ctx::next_timing_slot() {
    std::lock_guard<std::mutex> lk(timing_mu);
    if (!timing || stage_ev.empty()) return nullptr;
    cudaEvent_t* slot = &stage_ev[(size_t)(timing_batches % kTimingSlots) * kStageEvents];
    ++timing_batches;
    return slot;
}

vx_status vx_ctx_stage_times_detail(vx_ctx* ctx, float* census_ms, float* costs_ms, float* aggregate_ms,
                                    float* wta_ms) {
    if (!ctx) return fail(VX_ERR_INVALID_ARGUMENT, "vx_ctx_stage_times: ctx is NULL");
    DeviceGuard g(ctx->device);
    std::lock_guard<std::mutex> lk(ctx->timing_mu);
    const int n = std::min(ctx->timing_batches, (int)vx_ctx::kTimingSlots);
    if (ctx->stage_ev.empty() || n == 0)
        return fail(VX_ERR_NOT_READY, "vx_ctx_stage_times: no timed batch since timing was enabled");
    constexpr int kStages = vx_ctx::kStageEvents - 1;
    double sum[kStages] = {};
    for (int b = 0; b < n; ++b) {
        cudaEvent_t* ev = &ctx->stage_ev[(size_t)b * vx_ctx::kStageEvents];
        cudaError_t e = cudaEventSynchronize(ev[kStages]);
        for (int i = 0; i < kStages && e == cudaSuccess; ++i) {
            float t = 0;
            e = cudaEventElapsedTime(&t, ev[i], ev[i + 1]);
            sum[i] += t;
        }
        if (e != cudaSuccess) return cuda_fail(e, "reading stage timing events");
    }
    if (census_ms) *census_ms = (float)(sum[0] / n);
    if (costs_ms) *costs_ms = (float)(sum[1] / n);
    if (aggregate_ms) *aggregate_ms = (float)(sum[2] / n);
    if (wta_ms) *wta_ms = (float)(sum[3] / n);
    return VX_OK;
}

vx_status vx_ctx_stage_times(vx_ctx* ctx, float* census_ms, float* aggregate_ms, float* wta_ms) {
    float census = 0, costs = 0;
    vx_status st = vx_ctx_stage_times_detail(ctx, &census, &costs, aggregate_ms, wta_ms);
    if (st == VX_OK && census_ms) *census_ms = census + costs;
    return st;
}

vx_status vx_ctx_set_workspace_limit(vx_ctx* ctx, size_t bytes) {
    if (!ctx || bytes == 0) return fail(VX_ERR_INVALID_ARGUMENT, "vx_ctx_set_workspace_limit: bad argument");
    ctx->workspace_limit = bytes;
    return VX_OK;
}

vx_stream vx_ctx_stream(vx_ctx* ctx) { return ctx ? (vx_stream)ctx->stream : nullptr; }

vx_status vx_ctx_synchronize(vx_ctx* ctx) {
    if (!ctx) return fail(VX_ERR_INVALID_ARGUMENT, "vx_ctx_synchronize: ctx is NULL");
    DeviceGuard g(ctx->device);
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    return e == cudaSuccess ? VX_OK : cuda_fail(e, "vx_ctx_synchronize");
}

vx_status vx_image_create(vx_ctx* ctx, uint32_t width, uint32_t height, vx_format format,
                          vx_image** out) {
    if (!ctx || !out) return fail(VX_ERR_INVALID_ARGUMENT, "vx_image_create: NULL argument");
    *out = nullptr;
    const size_t eb = format_bytes(format);
    if (!eb) return fail(VX_ERR_INVALID_ARGUMENT, "vx_image_create: bad format %d", (int)format);
    if (width == 0 || height == 0)
        return fail(VX_ERR_INVALID_ARGUMENT, "vx_image_create: empty image %ux%u", width, height);
    DeviceGuard g(ctx->device);
    void* ptr = nullptr;
    size_t pitch = 0;
    count_alloc();
    cudaError_t e = cudaMallocPitch(&ptr, &pitch, (size_t)width * eb, height);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(VX_ERR_BUFFER_ALLOC, "buffer allocation failed (%zu bytes)",
                    (size_t)width * eb * height);
    }
    auto* img = new vx_image;
    img->ctx = ctx;
    img->ptr = ptr;
    img->pitch = pitch;
    img->width = width;
    img->height = height;
    img->format = format;
    img->owned = true;
    *out = img;
    return VX_OK;
}

vx_status vx_image_wrap_device(vx_ctx* ctx, void* device_ptr, size_t pitch_bytes, uint32_t width,
                               uint32_t height, vx_format format, vx_image** out) {
    if (!ctx || !out || !device_ptr)
        return fail(VX_ERR_INVALID_ARGUMENT, "vx_image_wrap_device: NULL argument");
    *out = nullptr;
    const size_t eb = format_bytes(format);
    if (!eb) return fail(VX_ERR_INVALID_ARGUMENT, "vx_image_wrap_device: bad format");
    if (width == 0 || height == 0 || pitch_bytes < width * eb)
        return fail(VX_ERR_INVALID_ARGUMENT, "vx_image_wrap_device: bad size/pitch");
    if (format != VX_FORMAT_U8 && (pitch_bytes % eb != 0 || (uintptr_t)device_ptr % eb != 0))
        return fail(VX_ERR_INVALID_ARGUMENT, "vx_image_wrap_device: misaligned plane");
    auto* img = new vx_image;
    img->ctx = ctx;
    img->ptr = device_ptr;
    img->pitch = pitch_bytes;
    img->width = width;
    img->height = height;
    img->format = format;
    img->owned = false;
    *out = img;
    return VX_OK;
}

void vx_image_destroy(vx_image* img) {
    if (!img) return;
    if (img->owned) {
        DeviceGuard g(img->ctx->device);
        cudaFree(img->ptr);
    }
    delete img;
}

uint32_t vx_image_width(const vx_image* img) { return img ? img->width : 0; }
uint32_t vx_image_height(const vx_image* img) { return img ? img->height : 0; }
void* vx_image_device_ptr(const vx_image* img) { return img ? img->ptr : nullptr; }
size_t vx_image_pitch(const vx_image* img) { return img ? img->pitch : 0; }

static vx_status copy_2d(const vx_image* img, void* dst, size_t dpitch, const void* src,
                         size_t spitch, cudaMemcpyKind kind, vx_stream stream) {
    DeviceGuard g(img->ctx->device);
    cudaStream_t s = stream ? (cudaStream_t)stream : img->ctx->stream;
    const size_t row = (size_t)img->width * format_bytes(img->format);
    cudaError_t e = cudaMemcpy2DAsync(dst, dpitch, src, spitch, row, img->height, kind, s);
    if (e == cudaSuccess && !stream) e = cudaStreamSynchronize(s);
    return e == cudaSuccess ? VX_OK : cuda_fail(e, "image copy");
}

vx_status vx_image_upload(vx_image* img, const void* host, size_t host_pitch, vx_stream stream) {
    if (!img || !host) return fail(VX_ERR_INVALID_ARGUMENT, "vx_image_upload: NULL argument");
    const size_t row = (size_t)img->width * format_bytes(img->format);
    if (host_pitch == 0) host_pitch = row;
    if (host_pitch < row) return fail(VX_ERR_INVALID_ARGUMENT, "vx_image_upload: pitch < row");
    return copy_2d(img, img->ptr, img->pitch, host, host_pitch, cudaMemcpyHostToDevice, stream);
}

vx_status vx_image_download(const vx_image* img, void* host, size_t host_pitch, vx_stream stream) {
    if (!img || !host) return fail(VX_ERR_INVALID_ARGUMENT, "vx_image_download: NULL argument");
    const size_t row = (size_t)img->width * format_bytes(img->format);
    if (host_pitch == 0) host_pitch = row;
    if (host_pitch < row) return fail(VX_ERR_INVALID_ARGUMENT, "vx_image_download: pitch < row");
    return copy_2d(img, host, host_pitch, img->ptr, img->pitch, cudaMemcpyDeviceToHost, stream);
}

}  // extern "C"
