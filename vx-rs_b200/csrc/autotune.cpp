// In-house autotuner of the aggregation launch shape.
//
// The path-aggregation kernel runs one CTA per SM holding 1..N warpgroups (each
// scanline is serial work: more warps per SM raise throughput until the
// longest scanlines, slowed by a crowded SM, dominate). The best count depends
// on the batch: its largest and smallest disparity counts (the scanline-pair
// kernel gives each warpgroup a TMEM budget for one disparity class, so a mix
// of D can hold more warpgroups than its largest D alone), its census word
// width and how many units it queues. Each candidate count is timed with the
// plan built for it (its queue classes order the units). vx_sgm_autotune_batch times every candidate on
// a real batch with CUDA events around the aggregation launch and records the
// fastest in the SGMStereo handle; later batches with the same key use it. The
// table is saved to / loaded from a small JSON file.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <vector>

#include "vx_internal.hpp"

namespace vxsgm {

TuneKey tune_key(const Plan& plan) {
    TuneKey k;
    k.dp_max = plan.dp_max;
    k.census64 = plan.census64 ? 1 : 0;
    k.units_log2 = plan.units32 <= 0 ? 0 : (int)std::floor(std::log2((double)plan.units32));
    k.wide = plan.wide_tiles ? 1 : 0;
    k.dp_min = plan.dp_min;
    return k;
}

}  // namespace vxsgm

using namespace vxsgm;

namespace {

// The planner proper: the plan in the autotuned form and launch shape.
vx_status plan_uncached(vx_sgm* sgm, const std::vector<PairSpec>& specs, Plan* plan) {
    vx_status st = build_plan(specs, plan);
    if (st != VX_OK) return st;
    vx_sgm::Tuned t{0, 0, 0.0f};
    {
        std::lock_guard<std::mutex> lk(sgm->tune_mu);
        auto it = sgm->tuned.find(tune_key(*plan));
        if (it != sgm->tuned.end()) t = it->second;
    }
    if (t.warpgroups == 0) return st;          // not tuned: the planner's heuristic
    int unit = t.unit_scanlines;
    if (std::getenv("VX_SGM_AGG_FORM")) unit = plan->unit_scanlines;   // the forced form wins
    if (unit != plan->unit_scanlines || t.warpgroups != plan->agg.warpgroups) {
        const int wg = unit == t.unit_scanlines ? t.warpgroups : 0;
        *plan = Plan();
        st = build_plan(specs, plan, unit, wg);
    }
    return st;
}

}  // namespace

vx_status vx_sgm::plan_batch(const std::vector<PairSpec>& specs, Plan* plan) {
    std::string key = bucket_key(specs);
    for (const auto& s : specs) key += s.compact_shadow ? 'c' : 'f';
    uint64_t version;
    {
        std::lock_guard<std::mutex> lk(tune_mu);
        version = tune_version;
    }
    {
        std::lock_guard<std::mutex> lk(plan_mu);
        for (auto& e : plans) {
            if (e.key != key || e.version != version) continue;
            for (const auto& s : specs) {          // formats, output sizes and pitches may differ
                const vx_status vs = validate_pair(s);
                if (vs != VX_OK) return vs;
            }
            *plan = e.plan;
            rebind_pointers(*plan, specs);
            e.last_use = ++plan_clock;
            return VX_OK;
        }
    }
    const vx_status st = plan_uncached(this, specs, plan);
    if (st != VX_OK) return st;
    std::lock_guard<std::mutex> lk(plan_mu);
    if (plans.size() >= kPlanCacheEntries) {
        auto lru = std::min_element(plans.begin(), plans.end(),
                                    [](const PlanEntry& a, const PlanEntry& b) { return a.last_use < b.last_use; });
        plans.erase(lru);
    }
    plans.push_back({key, version, *plan, ++plan_clock});
    return st;
}

extern "C" {

vx_status vx_sgm_autotune_batch(vx_sgm* sgm, vx_ctx* ctx, uint32_t n, const vx_image* const* left,
                                const vx_image* const* right, vx_image* const* out_f32,
                                vx_image* const* out_i16, const vx_sgm_config* cfgs,
                                uint32_t iterations, uint32_t* best_warpgroups, float* best_ms,
                                uint32_t* best_unit_scanlines) {
    if (!sgm || !ctx || !n || !left || !right || !out_f32 || !cfgs)
        return fail(VX_ERR_INVALID_ARGUMENT, "autotune_batch: NULL argument");
    if (iterations == 0) iterations = 1;
    std::vector<PairSpec> specs(n);
    for (uint32_t i = 0; i < n; ++i)
        specs[i] = {left[i], right[i], out_f32[i], out_i16 ? out_i16[i] : nullptr, cfgs[i]};
    DeviceGuard g(ctx->device);
    cudaEvent_t ev[vx_ctx::kStageEvents] = {};
    for (auto& x : ev) cudaEventCreate(&x);
    vx_status st = VX_OK;
    int best_w = 0, best_unit = 0;
    float best = 0.0f;
    TuneKey key{};
    // Every aggregation form (32-scanline units on the single-scanline kernel,
    // 64-scanline units on the scanline-pair kernel, the across-lanes scan
    // kernel), every launch shape of each.
    for (int unit : {32, kUnitScanlines, kScanForm}) {
        if (const char* f = std::getenv("VX_SGM_AGG_FORM")) {
            const int forced = std::strcmp(f, "single") == 0 ? 32
                             : std::strcmp(f, "pairs") == 0 ? kUnitScanlines
                             : std::strcmp(f, "scan") == 0 ? kScanForm : unit;
            if (unit != forced) continue;
        }
        Plan plan;
        st = build_plan(specs, &plan, unit);
        if (st != VX_OK) break;
        key = tune_key(plan);
        const size_t ws_bytes = plan.ws_bytes;   // the same for every launch shape
        char* ws = nullptr;
        count_alloc();
        cudaError_t e = cudaMallocFromPoolAsync(reinterpret_cast<void**>(&ws), ws_bytes, ctx->pool,
                                                ctx->stream);
        if (e != cudaSuccess) {
            cudaGetLastError();
            st = fail(VX_ERR_BUFFER_ALLOC, "buffer allocation failed (%zu bytes)", ws_bytes);
            break;
        }
        const int wmax = aggregate_max_warpgroups(plan.unit_scanlines, plan.dp_max, plan.dp_min, plan.census64,
                                                  plan.wide_tiles);
        for (int w = 1; w <= wmax && st == VX_OK; ++w) {
            // The plan of this launch shape (its queue classes order the units).
            Plan shaped;
            st = build_plan(specs, &shaped, unit, w);
            if (st != VX_OK) break;
            if (shaped.agg.warpgroups != w || shaped.ws_bytes != ws_bytes) continue;  // not a shape of its own
            bind_plan(shaped, ws);
            double total = 0.0;
            for (uint32_t it = 0; it <= iterations && st == VX_OK; ++it) {  // first run untimed
                st = run_plan(shaped, ws, ctx->stream, ev);
                if (st != VX_OK) break;
                e = cudaEventSynchronize(ev[4]);
                float ms = 0.0f;
                if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, ev[2], ev[3]);
                if (e != cudaSuccess) st = cuda_fail(e, "autotune timing");
                if (it > 0) total += ms;
            }
            const float mean = (float)(total / iterations);
            if (st == VX_OK && (best_w == 0 || mean < best)) {
                best_w = w;
                best_unit = unit;
                best = mean;
            }
        }
        cudaFreeAsync(ws, ctx->stream);
        cudaStreamSynchronize(ctx->stream);
    }
    for (auto& x : ev) cudaEventDestroy(x);
    if (st != VX_OK) return st;
    {
        std::lock_guard<std::mutex> lk(sgm->tune_mu);
        sgm->tuned[key] = {best_unit, best_w, best};
        ++sgm->tune_version;
    }
    if (best_warpgroups) *best_warpgroups = (uint32_t)best_w;
    if (best_ms) *best_ms = best;
    if (best_unit_scanlines) *best_unit_scanlines = (uint32_t)best_unit;
    return VX_OK;
}

vx_status vx_sgm_tuning_save(vx_sgm* sgm, const char* path) {
    if (!sgm || !path) return fail(VX_ERR_INVALID_ARGUMENT, "tuning_save: NULL argument");
    std::ofstream f(path);
    if (!f) return fail(VX_ERR_INVALID_ARGUMENT, "tuning_save: cannot open %s", path);
    std::lock_guard<std::mutex> lk(sgm->tune_mu);
    f << "{\"version\": 1, \"entries\": [";
    bool first = true;
    for (const auto& kv : sgm->tuned) {
        f << (first ? "" : ", ") << "{\"dp_max\": " << kv.first.dp_max << ", \"dp_min\": " << kv.first.dp_min
          << ", \"census64\": " << kv.first.census64 << ", \"units_log2\": " << kv.first.units_log2
          << ", \"wide\": " << kv.first.wide << ", \"unit_scanlines\": " << kv.second.unit_scanlines
          << ", \"warpgroups\": " << kv.second.warpgroups
          << ", \"aggregate_ms\": " << kv.second.aggregate_ms << "}";
        first = false;
    }
    f << "]}\n";
    return f.good() ? VX_OK : fail(VX_ERR_INVALID_ARGUMENT, "tuning_save: write failed");
}

// Reads the file written by vx_sgm_tuning_save (a flat list of entries with
// integer fields; anything else in the file is ignored).
vx_status vx_sgm_tuning_load(vx_sgm* sgm, const char* path) {
    if (!sgm || !path) return fail(VX_ERR_INVALID_ARGUMENT, "tuning_load: NULL argument");
    std::ifstream f(path);
    if (!f) return fail(VX_ERR_INVALID_ARGUMENT, "tuning_load: cannot open %s", path);
    std::stringstream ss;
    ss << f.rdbuf();
    const std::string text = ss.str();
    auto field = [&](size_t from, size_t to, const char* name, double* v) {
        const std::string key = std::string("\"") + name + "\":";
        size_t p = text.find(key, from);
        if (p == std::string::npos || p > to) return false;
        *v = std::strtod(text.c_str() + p + key.size(), nullptr);
        return true;
    };
    size_t pos = 0;
    int loaded = 0;
    std::lock_guard<std::mutex> lk(sgm->tune_mu);
    while ((pos = text.find('{', pos + 1)) != std::string::npos) {
        const size_t end = text.find('}', pos);
        if (end == std::string::npos) break;
        double dp, c64, ul, wg, ms = 0, wide = 0, us = 32;
        if (field(pos, end, "dp_max", &dp) && field(pos, end, "census64", &c64) &&
            field(pos, end, "units_log2", &ul) && field(pos, end, "warpgroups", &wg)) {
            field(pos, end, "aggregate_ms", &ms);
            field(pos, end, "wide", &wide);
            field(pos, end, "unit_scanlines", &us);
            double dmin = dp;   // files without dp_min: batches of one D
            field(pos, end, "dp_min", &dmin);
            if (wg >= 1 && dp >= 8 && dmin >= 8 && dmin <= dp && (us == 32 || us == kUnitScanlines || us == kScanForm)) {
                sgm->tuned[TuneKey{(int)dp, (int)c64, (int)ul, (int)wide, (int)dmin}] = {(int)us, (int)wg, (float)ms};
                ++sgm->tune_version;
                ++loaded;
            }
        }
        pos = end;
    }
    if (!loaded) return fail(VX_ERR_INVALID_CONFIG, "tuning_load: no entries in %s", path);
    return VX_OK;
}

}  // extern "C"
