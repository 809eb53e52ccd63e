// SGMStereo entry points of the vx_sgm C ABI (vx-vision/src/kernels/sgm.rs).
#include <cfloat>
#include <cstring>
#include <vector>

#include "vx_internal.hpp"

using namespace vxsgm;

namespace {

// Runs a batch; if keep_ws is non-null the workspace is handed back to the
// caller (who must free it with cudaFreeAsync) instead of being released.
vx_status run_batch(vx_sgm* sgm, vx_ctx* ctx, const std::vector<PairSpec>& specs,
                    cudaStream_t stream, bool synchronous, char** keep_ws, Plan* plan_out) {
    Plan plan;
    vx_status st = sgm->plan_batch(specs, &plan);
    if (st != VX_OK) return st;
    if (specs.empty()) return VX_OK;
    if (plan.ws_bytes > ctx->workspace_limit && specs.size() > 1 && !keep_ws) {
        // Staging: consecutive sub-batches that each fit the workspace limit run
        // one after another on the stream (each reuses the previous one's
        // workspace from the pool).
        std::vector<PairSpec> chunk;
        size_t bytes = 0;
        for (size_t i = 0; i <= specs.size(); ++i) {
            size_t b = 0;
            if (i < specs.size())
                b = vx_sgm_workspace_bytes(specs[i].left->width, specs[i].left->height, &specs[i].cfg) +
                    (64 << 10);
            if (i == specs.size() || (!chunk.empty() && bytes + b > ctx->workspace_limit)) {
                st = run_batch(sgm, ctx, chunk, stream, false, nullptr, nullptr);
                if (st != VX_OK) return st;
                chunk.clear();
                bytes = 0;
            }
            if (i < specs.size()) {
                chunk.push_back(specs[i]);
                bytes += b;
            }
        }
        if (synchronous) {
            cudaError_t e = cudaStreamSynchronize(stream);
            if (e != cudaSuccess) return cuda_fail(e, "SGM execution");
        }
        return VX_OK;
    }
    DeviceGuard g(ctx->device);
    char* ws = nullptr;
    count_alloc();
    cudaError_t e = cudaMallocFromPoolAsync(reinterpret_cast<void**>(&ws), plan.ws_bytes, ctx->pool, stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(VX_ERR_BUFFER_ALLOC, "buffer allocation failed (%zu bytes)", plan.ws_bytes);
    }
    bind_plan(plan, ws);
    st = run_plan(plan, ws, stream, ctx->next_timing_slot());
    if (keep_ws && st == VX_OK) {
        *keep_ws = ws;
    } else {
        cudaFreeAsync(ws, stream);
    }
    if (st == VX_OK && synchronous) {
        e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) st = cuda_fail(e, "SGM execution");
    }
    if (plan_out) *plan_out = std::move(plan);
    return st;
}

// A synchronous batch whose byte-slab pairs keep their escaped path vectors in
// a pool of 1/16 of their vectors instead of a full u16 shadow (about a third
// of the workspace), so that fewer, larger sub-batches fit the workspace limit.
// After each sub-batch the pairs' overflow flags come back; a pair whose pool
// ran out (more than 1/16 of its path vectors held a value above a byte) is
// recomputed with a full shadow at the end, so results never depend on the pool.
vx_status run_batch_pooled(vx_sgm* sgm, vx_ctx* ctx, const std::vector<PairSpec>& specs, cudaStream_t stream) {
    std::vector<PairSpec> pooled(specs);
    for (auto& s : pooled) s.compact_shadow = true;
    for (const auto& s : pooled) {
        const vx_status st = validate_pair(s);
        if (st != VX_OK) return st;
    }
    DeviceGuard g(ctx->device);
    std::vector<PairSpec> rerun;
    size_t i0 = 0;
    while (i0 < pooled.size()) {
        // The longest run of pairs from i0 whose pooled workspaces fit the limit (at least one).
        size_t i1 = i0, bytes = 0;
        while (i1 < pooled.size()) {
            const PairSpec& s = pooled[i1];
            const size_t ct = census_bits(s.cfg) > 32 ? 8 : 4;
            const size_t b = pair_workspace_bytes(s.left->width, s.left->height, s.cfg, ct, true) +
                             pair_cost_bytes(s.left->width, s.left->height, s.cfg) + (64 << 10);
            if (i1 > i0 && bytes + b > ctx->workspace_limit) break;
            bytes += b;
            ++i1;
        }
        const std::vector<PairSpec> chunk(pooled.begin() + i0, pooled.begin() + i1);
        Plan plan;
        vx_status st = sgm->plan_batch(chunk, &plan);
        if (st != VX_OK) return st;
        char* ws = nullptr;
        count_alloc();
        cudaError_t e = cudaMallocFromPoolAsync(reinterpret_cast<void**>(&ws), plan.ws_bytes, ctx->pool, stream);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(VX_ERR_BUFFER_ALLOC, "buffer allocation failed (%zu bytes)", plan.ws_bytes);
        }
        bind_plan(plan, ws);
        st = run_plan(plan, ws, stream, ctx->next_timing_slot());
        std::vector<uint32_t> esc(2 * chunk.size(), 0u);
        if (st == VX_OK) {
            e = cudaMemcpyAsync(esc.data(), ws + plan.off_escape(), esc.size() * sizeof(uint32_t),
                                cudaMemcpyDeviceToHost, stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
            if (e != cudaSuccess) st = cuda_fail(e, "SGM execution");
        }
        cudaFreeAsync(ws, stream);
        if (st != VX_OK) return st;
        for (size_t k = 0; k < chunk.size(); ++k)
            if (esc[2 * k + 1] != 0u) rerun.push_back(specs[i0 + k]);   // the pair as given: full shadow
        i0 = i1;
    }
    if (!rerun.empty()) return run_batch(sgm, ctx, rerun, stream, true, nullptr, nullptr);
    cudaError_t e = cudaStreamSynchronize(stream);
    return e == cudaSuccess ? VX_OK : cuda_fail(e, "SGM execution");
}

}  // namespace

namespace vxsgm {
vx_status run_batch_plain(vx_sgm* sgm, vx_ctx* ctx, const std::vector<PairSpec>& specs,
                          cudaStream_t stream) {
    return run_batch(sgm, ctx, specs, stream, false, nullptr, nullptr);
}
}  // namespace vxsgm

extern "C" {

void vx_sgm_config_default(vx_sgm_config* cfg) {
    if (!cfg) return;
    // SGMStereoConfig::default(), vx-vision/src/kernels/sgm.rs:39-49.
    cfg->num_disparities = 128;
    cfg->p1 = 10.0f;
    cfg->p2 = 120.0f;
    cfg->census_radius_x = 4;
    cfg->census_radius_y = 3;
    // Extensions, defaulting to the reference's behaviour.
    cfg->num_paths = 2;
    cfg->subpixel = 1;
    cfg->lr_check = 0;
    cfg->lr_tolerance = 1;
    cfg->invalid_value = -1.0f;
}

void vx_sgm_config_new(vx_sgm_config* cfg, uint32_t num_disparities) {
    vx_sgm_config_default(cfg);
    if (cfg) cfg->num_disparities = num_disparities;
}

vx_status vx_sgm_create(vx_ctx* ctx, vx_sgm** out) {
    if (!ctx || !out) return fail(VX_ERR_INVALID_ARGUMENT, "vx_sgm_create: NULL argument");
    *out = nullptr;
    DeviceGuard g(ctx->device);
    // The reference resolves and compiles its three pipelines here
    // (sgm.rs:73-105); the equivalent check is that this library's sm_100a
    // kernel images load on the device.
    cudaError_t e = prepare_wta_kernel();
    if (e == cudaSuccess) e = prepare_aggregate_kernels();
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(VX_ERR_SHADER_MISSING, "SGM kernels unavailable on device %d: %s", ctx->device,
                    cudaGetErrorString(e));
    }
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device) != cudaSuccess || sms <= 0) {
        cudaGetLastError();
        return fail(VX_ERR_PIPELINE_COMPILE, "no multiprocessors on device %d", ctx->device);
    }
    auto* s = new vx_sgm;
    s->ctx = ctx;
    *out = s;
    return VX_OK;
}

void vx_sgm_destroy(vx_sgm* sgm) { delete sgm; }

vx_status vx_sgm_compute_disparity(vx_sgm* sgm, vx_ctx* ctx, const vx_image* left,
                                   const vx_image* right, vx_image* out_f32, vx_image* out_i16,
                                   const vx_sgm_config* cfg, vx_stream stream) {
    if (!sgm || !ctx || !cfg) return fail(VX_ERR_INVALID_ARGUMENT, "compute_disparity: NULL argument");
    std::vector<PairSpec> specs{{left, right, out_f32, out_i16, *cfg}};
    cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
    if (sgm->graph_capacity) return run_batch_graph(sgm, ctx, specs, s, stream == nullptr);
    return run_batch(sgm, ctx, specs, s, stream == nullptr, nullptr, nullptr);
}

vx_status vx_sgm_compute(vx_sgm* sgm, vx_ctx* ctx, const vx_image* left, const vx_image* right,
                         const vx_sgm_config* cfg, const vx_camera_intrinsics* intrinsics,
                         float baseline, vx_image* depth_out, vx_depth_map* out) {
    if (!sgm || !ctx || !left || !right || !cfg || !intrinsics || !out)
        return fail(VX_ERR_INVALID_ARGUMENT, "compute: NULL argument");
    std::memset(out, 0, sizeof *out);
    // sgm.rs:278-287: an R32Float output of the left image's size, the disparity
    // computation, and a DepthMap over that texture (min 0, max f32::MAX).
    vx_image* disp = nullptr;
    vx_status st = vx_image_create(ctx, left->width, left->height, VX_FORMAT_F32, &disp);
    if (st != VX_OK) return st;
    std::vector<PairSpec> specs{{left, right, disp, nullptr, *cfg}};
    specs[0].out_depth = depth_out;
    specs[0].depth_scale = intrinsics->fx * baseline;
    specs[0].depth_invalid = 0.0f;
    st = run_batch(sgm, ctx, specs, ctx->stream, true, nullptr, nullptr);
    if (st != VX_OK) {
        vx_image_destroy(disp);
        return st;
    }
    out->texture = disp;
    out->intrinsics = *intrinsics;
    out->min_depth = 0.0f;
    out->max_depth = FLT_MAX;
    return VX_OK;
}

vx_status vx_sgm_compute_batch(vx_sgm* sgm, vx_ctx* ctx, uint32_t n, const vx_image* const* left,
                               const vx_image* const* right, vx_image* const* out_f32,
                               vx_image* const* out_i16, const vx_sgm_config* cfgs,
                               vx_stream stream) {
    if (!sgm || !ctx || (n && (!left || !right || !out_f32 || !cfgs)))
        return fail(VX_ERR_INVALID_ARGUMENT, "compute_batch: NULL argument");
    std::vector<PairSpec> specs(n);
    for (uint32_t i = 0; i < n; ++i)
        specs[i] = {left[i], right[i], out_f32[i], out_i16 ? out_i16[i] : nullptr, cfgs[i]};
    cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
    if (sgm->graph_capacity) {
        size_t total = 0;
        for (const auto& p : specs)
            if (p.left) total += vx_sgm_workspace_bytes(p.left->width, p.left->height, &p.cfg);
        if (total <= ctx->workspace_limit) return run_batch_graph(sgm, ctx, specs, s, stream == nullptr);
    }
    if (!stream) return run_batch_pooled(sgm, ctx, specs, s);   // synchronous: escape pools, exact re-runs
    return run_batch(sgm, ctx, specs, s, false, nullptr, nullptr);
}

size_t vx_sgm_workspace_bytes(uint32_t width, uint32_t height, const vx_sgm_config* cfg) {
    if (!cfg) return 0;
    return pair_workspace_bytes(width, height, *cfg, census_bits(*cfg) > 32 ? 8 : 4) +
           pair_cost_bytes(width, height, *cfg);
}

vx_status vx_sgm_debug_dump(vx_sgm* sgm, vx_ctx* ctx, const vx_image* left, const vx_image* right,
                            const vx_sgm_config* cfg, uint64_t* census_left,
                            uint64_t* census_right, uint16_t* path_costs, uint16_t* cost_volume) {
    if (!sgm || !ctx || !left || !cfg) return fail(VX_ERR_INVALID_ARGUMENT, "debug_dump: NULL argument");
    DeviceGuard g(ctx->device);
    vx_image* out = nullptr;
    vx_status st = vx_image_create(ctx, left->width, left->height, VX_FORMAT_F32, &out);
    if (st != VX_OK) return st;
    std::vector<PairSpec> specs{{left, right, out, nullptr, *cfg}};
    char* ws = nullptr;
    Plan plan;
    st = run_batch(sgm, ctx, specs, ctx->stream, true, &ws, &plan);
    if (st == VX_OK) {
        const PairDev& pd = plan.pairs[0];
        const size_t W = pd.width, H = pd.height, D = pd.nd, Dp = pd.nd_pad, P = pd.num_paths;
        const size_t npx = W * H;
        const size_t ct = plan.census64 ? 8 : 4;
        std::vector<uint8_t> cbuf(npx * ct);
        auto fetch_census = [&](const void* src, uint64_t* dst) {
            cudaMemcpy(cbuf.data(), src, npx * ct, cudaMemcpyDeviceToHost);
            for (size_t i = 0; i < npx; ++i) {
                uint64_t v = 0;
                std::memcpy(&v, cbuf.data() + i * ct, ct);
                dst[i] = v;
            }
        };
        if (census_left) fetch_census(pd.census_l, census_left);
        if (census_right) fetch_census(pd.census_r, census_right);
        if (path_costs || cost_volume) {
            const size_t Dv = pd.nd_vec;
            std::vector<uint8_t> slabs(pd.slab_stride * P + 1);
            std::vector<uint16_t> shadow(pd.shadow_stride * P);
            if (!pd.wide_slabs) cudaMemcpy(slabs.data(), pd.slabs, slabs.size() - 1, cudaMemcpyDeviceToHost);
            cudaMemcpy(shadow.data(), pd.shadow, shadow.size() * sizeof(uint16_t), cudaMemcpyDeviceToHost);
            if (cost_volume) std::memset(cost_volume, 0, npx * D * sizeof(uint16_t));
            for (size_t p = 0; p < P; ++p)
                for (size_t i = 0; i < npx; ++i) {
                    const uint8_t* vb = &slabs[p * pd.slab_stride + i * Dv];
                    const uint16_t* vs = &shadow[p * pd.shadow_stride + i * Dp];
                    const bool escaped = pd.wide_slabs || vb[0] == 0xFF;   // u16 values in the shadow
                    for (size_t d = 0; d < D; ++d) {
                        const uint16_t v = escaped ? vs[d] : vb[d];
                        if (path_costs) path_costs[(p * npx + i) * D + d] = v;
                        if (cost_volume) cost_volume[i * D + d] = (uint16_t)(cost_volume[i * D + d] + v);
                    }
                }
        }
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) st = cuda_fail(e, "debug dump copy");
        cudaFreeAsync(ws, ctx->stream);
        cudaStreamSynchronize(ctx->stream);
    }
    vx_image_destroy(out);
    return st;
}

}  // extern "C"
