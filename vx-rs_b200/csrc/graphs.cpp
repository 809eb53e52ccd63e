// CUDA graphs per shape bucket for the batched SGM path.
//
// A bucket is the ordered list of the pairs' sizes and configs. The first call
// of a bucket plans it, allocates a workspace that stays resident, uploads the
// plan tables and captures the launch sequence (counter reset, census,
// path aggregation, WTA) into a graph. Later calls of the same bucket only
// refresh the pair table (image and output pointers may differ) and launch
// the graph, skipping host planning and per-launch overhead. Buckets are kept
// in an LRU of vx_sgm::graph_capacity entries; an evicted bucket's workspace
// goes back to the context's pool. All calls of one bucket must be ordered on
// one stream (they share its workspace).
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <sstream>

#include "vx_internal.hpp"

namespace vxsgm {

std::string bucket_key(const std::vector<PairSpec>& specs) {
    std::ostringstream k;
    for (const auto& s : specs) {
        const vx_sgm_config& c = s.cfg;
        uint32_t p1, p2, inv;
        std::memcpy(&p1, &c.p1, 4);
        std::memcpy(&p2, &c.p2, 4);
        std::memcpy(&inv, &c.invalid_value, 4);
        k << s.left->width << 'x' << s.left->height << ':' << c.num_disparities << ',' << p1 << ','
          << p2 << ',' << c.census_radius_x << ',' << c.census_radius_y << ',' << c.num_paths
          << ',' << c.subpixel << ',' << c.lr_check << ',' << c.lr_tolerance << ',' << inv << ','
          << (s.out_i16 ? 1 : 0) << ',' << (s.out_depth ? 1 : 0) << ';';
    }
    // The planner's overrides of the slab format and the aggregation form
    // change the plan for the same shapes.
    for (const char* v : {"VX_SGM_SLAB_FORMAT", "VX_SGM_AGG_FORM", "VX_SGM_AGG_WARPGROUPS", "VX_SGM_SHADOW_POOL"})
        if (const char* e = std::getenv(v)) k << v << '=' << e << ';';
    return k.str();
}

namespace {

void destroy_entry(vx_sgm::GraphEntry* e, cudaStream_t stream) {
    if (e->exec) cudaGraphExecDestroy(e->exec);
    if (e->graph) cudaGraphDestroy(e->graph);
    for (auto ev : e->baked)
        if (ev) cudaEventDestroy(ev);
    if (e->ws) cudaFreeAsync(e->ws, stream);
    delete e;
}

// Refreshes the pointer fields of the bucket's pair table for this call.
}  // namespace

vx_status run_batch_graph(vx_sgm* sgm, vx_ctx* ctx, const std::vector<PairSpec>& specs,
                          cudaStream_t stream, bool synchronous) {
    for (const auto& s : specs) {
        vx_status st = validate_pair(s);
        if (st != VX_OK) return st;
    }
    if (specs.empty()) return VX_OK;
    DeviceGuard g(ctx->device);
    std::lock_guard<std::mutex> lk(sgm->graph_mu);
    const std::string key = bucket_key(specs);
    vx_sgm::GraphEntry* entry = nullptr;
    for (auto* e : sgm->graphs)
        if (e->key == key) entry = e;
    vx_status st = VX_OK;
    cudaError_t err = cudaSuccess;
    if (!entry) {
        auto* e = new vx_sgm::GraphEntry;
        e->key = key;
        st = sgm->plan_batch(specs, &e->plan);
        if (st == VX_OK) {
            count_alloc();
            err = cudaMallocFromPoolAsync(reinterpret_cast<void**>(&e->ws), e->plan.ws_bytes, ctx->pool,
                                          stream);
            if (err != cudaSuccess) {
                cudaGetLastError();
                e->ws = nullptr;
                st = fail(VX_ERR_BUFFER_ALLOC, "buffer allocation failed (%zu bytes)", e->plan.ws_bytes);
            }
        }
        if (st == VX_OK) {
            bind_plan(e->plan, e->ws);
            st = upload_plan(e->plan, e->ws, stream, false);
        }
        for (int i = 0; i < vx_ctx::kStageEvents && st == VX_OK; ++i) {
            err = cudaEventCreate(&e->baked[i]);
            if (err != cudaSuccess) st = cuda_fail(err, "graph timing events");
        }
        if (st == VX_OK) {
            err = cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal);
            if (err != cudaSuccess) st = cuda_fail(err, "beginning graph capture");
        }
        if (st == VX_OK) {
            const vx_status lst = launch_plan(e->plan, e->ws, stream, e->baked, true);
            err = cudaStreamEndCapture(stream, &e->graph);
            if (lst != VX_OK) st = lst;
            else if (err != cudaSuccess) st = cuda_fail(err, "ending graph capture");
        }
        if (st == VX_OK) {
            // The stage-timing event nodes, so each launch can point them at the
            // context's timing events.
            size_t num = 0;
            cudaGraphGetNodes(e->graph, nullptr, &num);
            std::vector<cudaGraphNode_t> nodes(num);
            cudaGraphGetNodes(e->graph, nodes.data(), &num);
            for (auto nd : nodes) {
                cudaGraphNodeType t;
                if (cudaGraphNodeGetType(nd, &t) != cudaSuccess || t != cudaGraphNodeTypeEventRecord)
                    continue;
                cudaEvent_t ev = nullptr;
                cudaGraphEventRecordNodeGetEvent(nd, &ev);
                for (int i = 0; i < vx_ctx::kStageEvents; ++i)
                    if (ev == e->baked[i]) e->ev_nodes[i] = nd;
            }
            err = cudaGraphInstantiate(&e->exec, e->graph, 0);
            if (err != cudaSuccess) st = cuda_fail(err, "instantiating the batch graph");
        }
        if (st != VX_OK) {
            destroy_entry(e, stream);
            return st;
        }
        sgm->graphs.push_back(e);
        entry = e;
        while (sgm->graphs.size() > sgm->graph_capacity) {  // evict least recently used
            auto lru = std::min_element(sgm->graphs.begin(), sgm->graphs.end(),
                                        [](auto* a, auto* b) { return a->last_use < b->last_use; });
            if (*lru == entry) break;
            destroy_entry(*lru, stream);
            sgm->graphs.erase(lru);
        }
    } else {
        rebind_pointers(entry->plan, specs);
        st = upload_plan(entry->plan, entry->ws, stream, true);
        if (st != VX_OK) return st;
    }
    entry->last_use = ++sgm->graph_clock;

    cudaEvent_t* slot = ctx->next_timing_slot();
    for (int i = 0; i < vx_ctx::kStageEvents; ++i)
        if (entry->ev_nodes[i])
            cudaGraphExecEventRecordNodeSetEvent(entry->exec, entry->ev_nodes[i],
                                                 slot ? slot[i] : entry->baked[i]);
    // census, the cost volume (scanline-pair form), aggregation, WTA
    count_launch(entry->plan.unit_scanlines != 32 ? 4 : 3);   // the cost volume in the pair and scan forms
    err = cudaGraphLaunch(entry->exec, stream);
    if (err != cudaSuccess) return cuda_fail(err, "launching the batch graph");
    if (synchronous) {
        err = cudaStreamSynchronize(stream);
        if (err != cudaSuccess) return cuda_fail(err, "SGM execution");
    }
    return VX_OK;
}

}  // namespace vxsgm

using namespace vxsgm;

vx_sgm::~vx_sgm() {
    for (auto* e : graphs) destroy_entry(e, ctx->stream);
    graphs.clear();
    cudaStreamSynchronize(ctx->stream);
}

extern "C" vx_status vx_sgm_set_graph_cache(vx_sgm* sgm, uint32_t max_buckets) {
    if (!sgm) return fail(VX_ERR_INVALID_ARGUMENT, "set_graph_cache: NULL handle");
    DeviceGuard g(sgm->ctx->device);
    std::lock_guard<std::mutex> lk(sgm->graph_mu);
    sgm->graph_capacity = max_buckets;
    while (sgm->graphs.size() > sgm->graph_capacity) {
        auto lru = std::min_element(sgm->graphs.begin(), sgm->graphs.end(),
                                    [](auto* a, auto* b) { return a->last_use < b->last_use; });
        destroy_entry(*lru, sgm->ctx->stream);
        sgm->graphs.erase(lru);
    }
    cudaStreamSynchronize(sgm->ctx->stream);
    return VX_OK;
}
