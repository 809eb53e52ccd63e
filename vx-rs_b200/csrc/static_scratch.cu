// Disparity computation that allocates no device memory.
//
// Some callers cannot allocate device memory at the moment they call in: a
// host application that reserves all GPU memory for its own allocator at
// start-up, a real-time loop that must not take the implicit device
// synchronisation cudaMalloc / cudaFree can cause, or a plugin whose host
// forbids allocation during a call. For them this entry point runs the same
// census -> path aggregation -> WTA kernels as vx_sgm_compute_disparity, but
// its intermediate state (plan tables, census words, per-path cost slabs)
// lives in one file-scope __device__ array of kStaticScratchBytes, so the call
// makes no cudaMalloc / cudaFree / pool allocation. The caller still provides
// the input and output planes.
//
// Costs and limits:
//  * The array occupies kStaticScratchBytes (64 MiB) on every GPU where this
//    library's module is loaded, until the process exits.
//  * A pair is accepted only if its whole workspace fits in the array
//    (vx_sgm_workspace_bytes plus a few KB of tables); larger pairs are
//    rejected with VX_ERR_BUDGET.
//  * All calls on a device share the one array, which keeps the last call's
//    contents: calls whose GPU work overlaps (different streams, or
//    different host threads without ordering) race on it. The work-queue
//    counters that must start at zero are cleared on the stream by every call.
//  * The first call on a device does the set-up for that device (the
//    scratch's device address via cudaGetSymbolAddress, the kernels'
//    shared-memory limits); make that first call before any stream capture.
#include <cuda_runtime.h>

#include <mutex>
#include <vector>

#include "vx_internal.hpp"

namespace vxsgm {
namespace {

constexpr size_t kStaticScratchBytes = 64ull << 20;
constexpr int kMaxDevices = 64;

__device__ __align__(256) unsigned char g_sgm_static_scratch[kStaticScratchBytes];

// Device address of g_sgm_static_scratch per device (host code must not use
// the symbol itself as an address: it is a host-side stand-in).
std::mutex g_setup_mu;
char* g_scratch_addr[kMaxDevices] = {};

vx_status scratch_for_current_device(char** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "no current CUDA device");
    if (dev < 0 || dev >= kMaxDevices)
        return fail(VX_ERR_DEVICE_NOT_FOUND, "device ordinal %d unsupported", dev);
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_sgm_static_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "locating the static scratch on the device");
        e = prepare_wta_kernel();
        if (e == cudaSuccess) e = prepare_aggregate_kernels();
        if (e != cudaSuccess) return cuda_fail(e, "configuring the SGM kernels");
        g_scratch_addr[dev] = static_cast<char*>(p);
    }
    *out = g_scratch_addr[dev];
    return VX_OK;
}

}  // namespace
}  // namespace vxsgm

using namespace vxsgm;

extern "C" size_t vx_sgm_static_scratch_bytes(void) { return kStaticScratchBytes; }

extern "C" vx_status vx_sgm_compute_disparity_noalloc(
    const uint8_t* left, size_t left_pitch, const uint8_t* right, size_t right_pitch,
    uint32_t width, uint32_t height, float* out_f32, size_t out_f32_pitch, int16_t* out_i16,
    size_t out_i16_pitch, const vx_sgm_config* cfg, vx_stream stream) {
    if (!left || !right || !out_f32 || !cfg)
        return fail(VX_ERR_INVALID_ARGUMENT, "compute_disparity_noalloc: NULL argument");
    if (width == 0 || height == 0)
        return fail(VX_ERR_INVALID_ARGUMENT, "compute_disparity_noalloc: empty image");
    if (left_pitch < width || right_pitch < width || out_f32_pitch < width * sizeof(float) ||
        (out_i16 && out_i16_pitch < width * sizeof(int16_t)))
        return fail(VX_ERR_INVALID_ARGUMENT, "compute_disparity_noalloc: pitch smaller than a row");
    // The WTA kernel stores whole floats and int16s: a plane or pitch that is not
    // a multiple of the element size would make it store to misaligned addresses
    // (the same rule vx_image_wrap_device applies to caller-owned planes).
    if ((uintptr_t)out_f32 % sizeof(float) != 0 || out_f32_pitch % sizeof(float) != 0 ||
        (out_i16 && ((uintptr_t)out_i16 % sizeof(int16_t) != 0 || out_i16_pitch % sizeof(int16_t) != 0)))
        return fail(VX_ERR_INVALID_ARGUMENT,
                    "compute_disparity_noalloc: misaligned output plane (F32 planes and pitches must be "
                    "multiples of 4 bytes, I16 ones of 2)");

    // Plain descriptors of the caller's planes (no device allocation behind them).
    vx_image l{}, r{}, of{}, oi{};
    l = {nullptr, const_cast<uint8_t*>(left), left_pitch, width, height, VX_FORMAT_U8, false};
    r = {nullptr, const_cast<uint8_t*>(right), right_pitch, width, height, VX_FORMAT_U8, false};
    of = {nullptr, out_f32, out_f32_pitch, width, height, VX_FORMAT_F32, false};
    oi = {nullptr, out_i16, out_i16_pitch, width, height, VX_FORMAT_I16, false};
    std::vector<PairSpec> specs{{&l, &r, &of, out_i16 ? &oi : nullptr, *cfg}};

    Plan plan;
    vx_status st = build_plan(specs, &plan);
    if (st != VX_OK) return st;
    if (plan.ws_bytes > kStaticScratchBytes)
        return fail(VX_ERR_BUDGET,
                    "compute_disparity_noalloc: this pair needs %zu bytes of scratch, the static "
                    "scratch holds %zu (use vx_sgm_compute_disparity for larger pairs)",
                    plan.ws_bytes, kStaticScratchBytes);
    char* base = nullptr;
    st = scratch_for_current_device(&base);
    if (st != VX_OK) return st;
    bind_plan(plan, base);
    cudaStream_t s = stream ? (cudaStream_t)stream : (cudaStream_t)0;
    st = run_plan(plan, base, s);
    if (st == VX_OK && !stream) {
        cudaError_t e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) st = cuda_fail(e, "SGM execution");
    }
    return st;
}
