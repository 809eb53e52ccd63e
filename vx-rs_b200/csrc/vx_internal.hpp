// Internal host-side definitions of the vx_sgm C ABI implementation.
#pragma once
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdint>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/vx_sgm.h"
#include "kernels.cuh"
#include "launch.hpp"

// The reference's Context (vx-vision/src/context.rs:17): device + queue.
// Here: a CUDA device, one stream and a stream-ordered memory pool whose
// release threshold keeps freed blocks cached, so steady-state calls do not
// reach the driver allocator.
struct vx_ctx {
    int device = 0;
    int sm_count = 0;
    cudaStream_t stream = nullptr;
    cudaMemPool_t pool = nullptr;
    // Largest workspace one batch may take; larger batches run as sequential
    // sub-batches (set at creation to 85% of the free device memory).
    size_t workspace_limit = 0;
    // Stage timing: per batch, 4 events bracket census | aggregation | WTA.
    // Batches since the last enable take consecutive slots of the ring.
    static constexpr int kTimingSlots = 256;
    static constexpr int kStageEvents = 5;  // before census, cost volume, aggregation, WTA; after WTA
    bool timing = false;
    int timing_batches = 0;
    std::vector<cudaEvent_t> stage_ev;  // kTimingSlots * kStageEvents when enabled
    std::mutex timing_mu;
    cudaEvent_t* next_timing_slot();
};

// The reference's Texture (vx-vision/src/texture.rs:29): a pitched 2D plane.
struct vx_image {
    vx_ctx* ctx = nullptr;
    void* ptr = nullptr;
    size_t pitch = 0;  // bytes
    uint32_t width = 0, height = 0;
    vx_format format = VX_FORMAT_U8;
    bool owned = false;
};

namespace vxsgm {

// Records a message for vx_last_error() on this host thread and returns status.
vx_status fail(vx_status status, const char* fmt, ...);
vx_status cuda_fail(cudaError_t err, const char* what);

// Makes ctx->device current for the scope of a call.
class DeviceGuard {
  public:
    explicit DeviceGuard(int device) {
        cudaGetDevice(&prev_);
        if (prev_ != device) cudaSetDevice(device);
        restore_ = prev_ != device;
    }
    ~DeviceGuard() {
        if (restore_) cudaSetDevice(prev_);
    }

  private:
    int prev_ = 0;
    bool restore_ = false;
};

size_t format_bytes(vx_format f);

// Validated description of one pair of a batch.
struct PairSpec {
    const vx_image* left;
    const vx_image* right;
    vx_image* out_f32;
    vx_image* out_i16;
    vx_sgm_config cfg;
    vx_image* out_depth = nullptr;  // optional: fx * baseline / disparity
    float depth_scale = 0.0f;
    float depth_invalid = 0.0f;
    // Byte-slab pairs only: escaped vectors go to a pool of
    // shadow_pool_vectors() instead of a full shadow (a third of the
    // workspace); the caller must check the pair's overflow flag after the run
    // and recompute it with a full shadow if it is set (the server does).
    bool compact_shadow = false;
};

// Vectors in a compact shadow pool: 1/16 of the pair's path-pixel vectors (at
// least 1024); VX_SGM_SHADOW_POOL=<n> sets it (tests force overflows with it).
uint32_t shadow_pool_vectors(uint32_t width, uint32_t height, const vx_sgm_config& cfg);

vx_status validate_pair(const PairSpec& p);
int census_bits(const vx_sgm_config& cfg);
bool wide_slabs(const vx_sgm_config& cfg);

// Host-side plan of one batched launch sequence (planner.cpp).
struct Plan {
    std::vector<PairDev> pairs;     // pointers relative to the workspace base until bound
    std::vector<JobDev> jobs;
    std::vector<UnitDev> units;     // all (pair, path, scanline-group) units, longest first
    bool census64 = false;
    bool wide_tiles = false;        // some pair has wide (u16) slabs
    bool compact = false;           // some pair has a shadow pool (shadow_cap > 0)
    int unit_scanlines = 32;        // 64: scanline-pair kernel, 32: single-scanline kernel
    long long units32 = 0;          // units the plan has at 32 scanlines (tuning key)
    int dp_max = 8;                 // largest padded disparity count
    int dp_min = 8;                 // smallest padded disparity count
    int total_tiles = 0, total_rows = 0, max_width = 0, max_rx = 0, max_ry = 0;
    AggLaunch agg;                  // aggregation launch shape and its queue classes (units ordered for it)
    // Workspace layout (byte offsets from the workspace base). The counter block
    // holds kMaxQueueClasses work-queue counters, then per pair the escape pool's
    // taken count and overflow flag (all cleared by every launch).
    size_t off_pairs = 0, off_jobs = 0, off_units = 0, off_counters = 0, off_data = 0;
    size_t ws_bytes = 0;
    std::vector<size_t> pair_data_off;  // per pair: census + slabs
    size_t off_escape() const { return off_counters + kMaxQueueClasses * sizeof(unsigned); }
    size_t counter_bytes() const { return sizeof(unsigned) * (kMaxQueueClasses + 2 * pairs.size()); }
};

// unit_scanlines: 32 or 64 forces the aggregation form (the autotuner's
// choice); 0 picks it from the amount of work. warpgroups: aggregation CTA
// size (the autotuner's choice, clamped to what an SM holds); 0 picks it from
// the batch. The unit queue is ordered for the chosen shape.
vx_status build_plan(const std::vector<PairSpec>& specs, Plan* plan, int unit_scanlines = 0, int warpgroups = 0);
// Workspace bytes of one pair's census planes and path slabs with census words
// of census_word_bytes (a batch uses 8-byte words for all its pairs as soon as
// one needs them), and an upper bound of its share of the plan tables.
// compact_shadow: the escape shadow is a pool (byte-slab pairs only).
size_t pair_workspace_bytes(uint32_t width, uint32_t height, const vx_sgm_config& cfg,
                            size_t census_word_bytes, bool compact_shadow = false);
size_t pair_table_bytes_bound(uint32_t width, uint32_t height, const vx_sgm_config& cfg);
// Bytes of a pair's matching-cost volume (batches run by the scanline-pair kernel).
size_t pair_cost_bytes(uint32_t width, uint32_t height, const vx_sgm_config& cfg);
// Points plan.pairs at the images and outputs of specs (same sizes and order
// as the specs the plan was built from).
void rebind_pointers(Plan& plan, const std::vector<PairSpec>& specs);
// Key of a batch's shapes: every pair's size and config in order, the output
// kinds and the planner's environment overrides (graphs.cpp).
std::string bucket_key(const std::vector<PairSpec>& specs);
// Resolves the workspace-relative pointers of plan.pairs against `base`.
void bind_plan(Plan& plan, char* base);
// Issues the whole batch (census, cost volume, aggregation, WTA) on `stream`
// with the workspace at `base` (plan must be bound to it).
// stage_events: null, or vx_ctx::kStageEvents events recorded before census,
// before the cost volume, before aggregation, before WTA and after WTA.
vx_status run_plan(const Plan& plan, char* base, cudaStream_t stream, cudaEvent_t* stage_events = nullptr);
// The two halves of run_plan: copy the plan tables into the workspace (all of
// them, or the pair table alone), and the launch sequence itself (which is
// what a CUDA graph of the batch captures).
vx_status upload_plan(const Plan& plan, char* base, cudaStream_t stream, bool pairs_only);
vx_status launch_plan(const Plan& plan, char* base, cudaStream_t stream, cudaEvent_t* stage_events,
                      bool capturing);

// Autotuning key of a batch: the best aggregation form and launch shape depend
// on the largest and smallest padded D (the TMEM budgets), the census word
// width, the tile format and the amount of queued work (log2 of its
// 32-scanline units).
struct TuneKey {
    int dp_max;
    int census64;
    int units_log2;
    int wide;
    int dp_min;
    bool operator<(const TuneKey& o) const {
        if (dp_max != o.dp_max) return dp_max < o.dp_max;
        if (dp_min != o.dp_min) return dp_min < o.dp_min;
        if (census64 != o.census64) return census64 < o.census64;
        if (wide != o.wide) return wide < o.wide;
        return units_log2 < o.units_log2;
    }
};
TuneKey tune_key(const Plan& plan);

}  // namespace vxsgm

struct vx_sgm;
namespace vxsgm {
// The batch without graphs, asynchronous on `stream` (workspace from the pool).
vx_status run_batch_plain(vx_sgm* sgm, vx_ctx* ctx, const std::vector<PairSpec>& specs,
                          cudaStream_t stream);
// The batch through the sgm's CUDA-graph cache (graphs.cpp).
vx_status run_batch_graph(vx_sgm* sgm, vx_ctx* ctx, const std::vector<PairSpec>& specs,
                          cudaStream_t stream, bool synchronous);
}  // namespace vxsgm

// The reference's SGMStereo (vx-vision/src/kernels/sgm.rs:62), plus the
// autotuned launch shapes of the batches it has seen.
struct vx_sgm {
    vx_ctx* ctx = nullptr;
    struct Tuned {
        int unit_scanlines;   // aggregation form: 32 single-scanline, 64 scanline pairs
        int warpgroups;
        float aggregate_ms;
    };
    std::mutex tune_mu;
    std::map<vxsgm::TuneKey, Tuned> tuned;
    uint64_t tune_version = 0;      // bumped whenever `tuned` changes (under tune_mu)
    // Plans of recent batch shapes, unbound (workspace offsets), so that a call
    // with the shapes of an earlier one skips the planner: the pair table's
    // pointers are refreshed and the pairs validated again. Keyed by the bucket
    // key, the pairs' shadow kinds and the tuning table's version.
    struct PlanEntry {
        std::string key;
        uint64_t version;
        vxsgm::Plan plan;
        uint64_t last_use;
    };
    static constexpr size_t kPlanCacheEntries = 16;
    std::mutex plan_mu;
    std::vector<PlanEntry> plans;
    uint64_t plan_clock = 0;
    // Plan of a batch in the autotuned form and launch shape (the planner's
    // heuristic when the batch's key was not tuned).
    vx_status plan_batch(const std::vector<vxsgm::PairSpec>& specs, vxsgm::Plan* plan);

    // CUDA graphs per shape bucket (see graphs.cpp): a bucket is the list of
    // every pair's size and config; image pointers may differ between calls.
    struct GraphEntry {
        std::string key;
        vxsgm::Plan plan;           // bound to ws
        char* ws = nullptr;         // resident workspace of the bucket
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        cudaEvent_t baked[vx_ctx::kStageEvents] = {};  // events the stage-timing nodes were captured with
        cudaGraphNode_t ev_nodes[vx_ctx::kStageEvents] = {};
        uint64_t last_use = 0;
    };
    std::mutex graph_mu;
    size_t graph_capacity = 0;
    uint64_t graph_clock = 0;
    std::vector<GraphEntry*> graphs;
    ~vx_sgm();
};
