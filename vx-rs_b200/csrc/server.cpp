// Serving loop: continuous batching of stereo requests under a device-memory
// budget (no counterpart in vx-vision, whose SGM call is one synchronous pair,
// vx-vision/src/kernels/sgm.rs:108-265).
//
// Memory is owned up front, so that steady-state serving never reaches a
// driver allocator (growing a memory pool or pinning host pages takes
// milliseconds to seconds and stalls every stream):
//  * a device arena of exactly the budget, taken from the context's pool when
//    the server starts; each batch occupies one block of it (its requests'
//    images and outputs, then the batch workspace: plan tables, census planes,
//    path slabs), placed first-fit and released when the batch retires;
//  * a pinned host staging arena (images in, disparities out), one block per
//    request from submit() to the wait() that returns its result; requests
//    beyond it fall back to individually pinned buffers.
// Requests are submitted from any host thread. A scheduler thread
//  * retires batches whose completion event has fired (results are already in
//    the request's pinned output buffer),
//  * admits pending requests in arrival order while the upper bound of their
//    device bytes fits the largest free block of the arena, up to max_batch per
//    batch, as soon as one of max_inflight stream slots is free, and
//  * launches the batch on that slot's stream: H2D of the images, the batched
//    SGM (census, one persistent aggregation launch, WTA), D2H of the
//    disparities and of the pairs' escape-pool flags, completion event.
// A request's workspace holds its escaped path vectors (values above a byte,
// rare) in a pool of 1/16 of its vectors instead of a full u16 shadow, which
// cuts the device bytes a request reserves by about 3x and so lets three times
// as many requests share a batch. A pair whose pool ran out is recomputed at
// the head of the queue with a full shadow (or fails with VX_ERR_BUDGET if that
// does not fit the budget), so results never depend on the pool.
// Batches on different slots overlap on the GPU, so requests that arrive while
// others run join the next batch instead of waiting for the GPU to drain. Each
// request's result does not depend on which other requests share its batch.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <thread>
#include <unordered_map>

#include "vx_internal.hpp"

namespace vxsgm {
namespace {

using Clock = std::chrono::steady_clock;

double ms_since(Clock::time_point t0, Clock::time_point t1) {
    return std::chrono::duration<double, std::milli>(t1 - t0).count();
}

constexpr size_t kBlockAlign = 256;
constexpr size_t kNoBlock = ~(size_t)0;
inline size_t block_align(size_t v) { return (v + kBlockAlign - 1) / kBlockAlign * kBlockAlign; }

// First-fit allocator over the offsets [0, capacity) of a buffer owned by the
// caller: address-ordered free blocks, merged with their neighbours on
// release. Sizes are rounded up to kBlockAlign.
class RangeAllocator {
  public:
    void reset(size_t capacity) {
        free_.clear();
        capacity_ = capacity / kBlockAlign * kBlockAlign;
        if (capacity_) free_[0] = capacity_;
        used_ = 0;
    }
    size_t alloc(size_t bytes) {
        bytes = block_align(std::max<size_t>(bytes, 1));
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < bytes) continue;
            const size_t off = it->first, rest = it->second - bytes;
            free_.erase(it);
            if (rest) free_[off + bytes] = rest;
            used_ += bytes;
            return off;
        }
        return kNoBlock;
    }
    void release(size_t off, size_t bytes) {
        bytes = block_align(std::max<size_t>(bytes, 1));
        used_ -= bytes;
        auto next = free_.lower_bound(off);
        if (next != free_.end() && off + bytes == next->first) {
            bytes += next->second;
            next = free_.erase(next);
        }
        if (next != free_.begin()) {
            auto prev = std::prev(next);
            if (prev->first + prev->second == off) {
                prev->second += bytes;
                return;
            }
        }
        free_[off] = bytes;
    }
    size_t largest() const {
        size_t m = 0;
        for (const auto& kv : free_) m = std::max(m, kv.second);
        return m;
    }
    size_t used() const { return used_; }
    size_t capacity() const { return capacity_; }

  private:
    std::map<size_t, size_t> free_;  // offset -> size
    size_t capacity_ = 0, used_ = 0;
};

enum ReqState { kPending, kRunning, kDone, kCancelled, kFailed };

struct Request {
    uint64_t id = 0;
    uint32_t w = 0, h = 0;
    vx_sgm_config cfg{};
    bool want_i16 = false;
    // Pinned staging: left and right (w*h each), then the f32 disparity (w*h),
    // then the i16 disparity (w*h) if wanted.
    char* host = nullptr;
    size_t host_off = kNoBlock;  // block of the staging arena, or kNoBlock (own pinned buffer)
    size_t host_bytes = 0;
    size_t dev_bytes = 0;        // upper bound of the request's share of a batch block
    bool full_shadow = false;    // recomputed after its escape pool ran out
    Clock::time_point t_submit, t_done;
    ReqState state = kPending;
    vx_status status = VX_OK;

    size_t px() const { return (size_t)w * h; }
    char* host_in() const { return host; }
    char* host_out() const { return host + 2 * px(); }
    size_t out_bytes() const { return 4 * px() + (want_i16 ? 2 * px() : 0); }
};

struct Slot {
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    std::vector<Request*> reqs;
    bool busy = false;
    size_t block_off = kNoBlock, block_bytes = 0;  // the batch's block of the device arena
    uint32_t* esc_host = nullptr;  // pinned: per request (escape count, pool overflow flag)
};

// Device bytes of a request's images and outputs inside a batch block.
size_t buffer_bytes(uint32_t w, uint32_t h, bool i16) {
    const size_t px = (size_t)w * h;
    return block_align(4 * px) + (i16 ? block_align(2 * px) : 0) + 2 * block_align(px);
}

}  // namespace
}  // namespace vxsgm

using namespace vxsgm;

struct vx_sgm_server {
    vx_sgm* sgm = nullptr;
    vx_ctx* ctx = nullptr;
    size_t budget = 0;
    uint32_t max_batch = 0;
    std::vector<Slot> slots;
    char* dev_arena = nullptr;
    RangeAllocator dev_alloc;        // scheduler thread only
    char* host_arena = nullptr;
    RangeAllocator host_alloc;       // under mu

    std::mutex mu;
    std::condition_variable cv_work;  // new submissions / stop
    std::condition_variable cv_done;  // a request finished
    std::deque<Request*> pending;
    std::unordered_map<uint64_t, std::unique_ptr<Request>> requests;
    uint64_t next_id = 1;
    bool stop = false;
    vx_server_stats stats{};
    std::thread worker;

    // Upper bound of the device bytes a request adds to a batch block: its
    // buffers, its workspace with 8-byte census words (a batch takes those for
    // all pairs when one pair needs them) and its share of the plan tables.
    static size_t request_bytes(uint32_t w, uint32_t h, const vx_sgm_config& cfg, bool i16, bool compact) {
        return buffer_bytes(w, h, i16) + pair_workspace_bytes(w, h, cfg, 8, compact) +
               pair_cost_bytes(w, h, cfg) + pair_table_bytes_bound(w, h, cfg);
    }

    bool host_get(Request* r);
    void host_put(Request* r);
    void run();
    void retire(Slot& s);
    void launch(Slot& s, std::vector<Request*>& batch);
};

bool vx_sgm_server::host_get(Request* r) {
    r->host_bytes = 2 * r->px() + r->out_bytes();
    {
        std::lock_guard<std::mutex> lk(mu);
        const size_t off = host_alloc.alloc(r->host_bytes);
        if (off != kNoBlock) {
            r->host_off = off;
            r->host = host_arena + off;
            return true;
        }
    }
    // Staging arena full: pin a buffer for this request alone (slow path).
    const auto t0 = Clock::now();
    void* p = nullptr;
    count_alloc();
    if (cudaMallocHost(&p, r->host_bytes) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    const uint64_t us = (uint64_t)(ms_since(t0, Clock::now()) * 1e3);
    std::lock_guard<std::mutex> lk(mu);
    stats.max_pinned_alloc_us = std::max(stats.max_pinned_alloc_us, us);
    stats.pinned_bytes += r->host_bytes;
    ++stats.staging_overflows;
    r->host = static_cast<char*>(p);
    r->host_off = kNoBlock;
    return true;
}

// Caller holds mu.
void vx_sgm_server::host_put(Request* r) {
    if (!r->host) return;
    if (r->host_off != kNoBlock) {
        host_alloc.release(r->host_off, r->host_bytes);
    } else {
        cudaFreeHost(r->host);
        stats.pinned_bytes -= r->host_bytes;
    }
    r->host = nullptr;
}

void vx_sgm_server::retire(Slot& s) {
    const auto now = Clock::now();
    if (s.block_off != kNoBlock) dev_alloc.release(s.block_off, s.block_bytes);
    s.block_off = kNoBlock;
    std::lock_guard<std::mutex> lk(mu);
    // Pairs whose escape pool ran out go back to the head of the queue, in
    // their order, with a full shadow.
    for (size_t i = s.reqs.size(); i-- > 0;) {
        Request* r = s.reqs[i];
        if (r->state != kRunning || r->full_shadow || s.esc_host[2 * i + 1] == 0) continue;
        r->full_shadow = true;
        r->dev_bytes = request_bytes(r->w, r->h, r->cfg, r->want_i16, false);
        ++stats.shadow_reruns;
        if (r->dev_bytes > budget) {
            r->state = kFailed;
            r->status = VX_ERR_BUDGET;
            r->t_done = now;
            ++stats.failed;
        } else {
            r->state = kPending;
            pending.push_front(r);
        }
    }
    stats.queued = pending.size();
    for (Request* r : s.reqs) {
        if (r->state == kPending) continue;  // queued again above
        r->t_done = now;
        if (r->state == kRunning) {
            r->state = kDone;
            ++stats.completed;
            stats.completed_pixel_disparities +=
                (uint64_t)r->w * r->h * r->cfg.num_disparities;
        }
    }
    stats.inflight_bytes = dev_alloc.used();
    s.reqs.clear();
    s.busy = false;
    cv_done.notify_all();
}

void vx_sgm_server::launch(Slot& s, std::vector<Request*>& batch) {
    DeviceGuard g(ctx->device);
    const size_t n = batch.size();
    // Images and outputs of each request inside the block, in order: f32
    // output, i16 output (if wanted), left, right. Their addresses are set once
    // the block is placed; the plan is sized first with the same shapes.
    std::vector<vx_image> imgs(n * 4);
    std::vector<PairSpec> specs;
    std::vector<size_t> buf_off(n);
    size_t buf_total = 0;
    for (size_t i = 0; i < n; ++i) {
        Request* r = batch[i];
        vx_image* im = &imgs[4 * i];
        im[0] = {ctx, nullptr, r->w, r->w, r->h, VX_FORMAT_U8, false};
        im[1] = {ctx, nullptr, r->w, r->w, r->h, VX_FORMAT_U8, false};
        im[2] = {ctx, nullptr, (size_t)r->w * 4, r->w, r->h, VX_FORMAT_F32, false};
        im[3] = {ctx, nullptr, (size_t)r->w * 2, r->w, r->h, VX_FORMAT_I16, false};
        specs.push_back({&im[0], &im[1], &im[2], r->want_i16 ? &im[3] : nullptr, r->cfg});
        specs.back().compact_shadow = !r->full_shadow;
        buf_off[i] = buf_total;
        buf_total += buffer_bytes(r->w, r->h, r->want_i16);
    }
    Plan plan;
    vx_status st = sgm->plan_batch(specs, &plan);
    if (st == VX_OK) {
        s.block_bytes = buf_total + plan.ws_bytes;
        s.block_off = dev_alloc.alloc(s.block_bytes);
        // Admission reserved an upper bound of this inside one free block.
        if (s.block_off == kNoBlock)
            st = fail(VX_ERR_BUFFER_ALLOC, "server: batch block of %zu bytes does not fit the arena",
                      s.block_bytes);
    }
    if (st == VX_OK) {
        char* block = dev_arena + s.block_off;
        for (size_t i = 0; i < n; ++i) {
            Request* r = batch[i];
            const size_t px = r->px();
            char* of = block + buf_off[i];
            char* oi = of + block_align(4 * px);
            char* li = oi + (r->want_i16 ? block_align(2 * px) : 0);
            char* ri = li + block_align(px);
            vx_image* im = &imgs[4 * i];
            im[0].ptr = li;
            im[1].ptr = ri;
            im[2].ptr = of;
            im[3].ptr = oi;
            cudaError_t e = cudaMemcpyAsync(li, r->host_in(), px, cudaMemcpyHostToDevice, s.stream);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(ri, r->host_in() + px, px, cudaMemcpyHostToDevice, s.stream);
            if (e != cudaSuccess) {
                st = cuda_fail(e, "server: image upload");
                break;
            }
        }
    }
    if (st == VX_OK) {
        char* ws = dev_arena + s.block_off + buf_total;
        rebind_pointers(plan, specs);
        bind_plan(plan, ws);
        st = run_plan(plan, ws, s.stream, ctx->next_timing_slot());
        if (st == VX_OK) {
            cudaError_t e = cudaMemcpyAsync(s.esc_host, ws + plan.off_escape(),
                                            2 * n * sizeof(uint32_t), cudaMemcpyDeviceToHost, s.stream);
            if (e != cudaSuccess) st = cuda_fail(e, "server: escape flags download");
        }
    }
    for (size_t i = 0; i < n && st == VX_OK; ++i) {
        Request* r = batch[i];
        const size_t px = r->px();
        char* of = dev_arena + s.block_off + buf_off[i];
        cudaError_t e = cudaMemcpyAsync(r->host_out(), of, 4 * px, cudaMemcpyDeviceToHost, s.stream);
        if (e == cudaSuccess && r->want_i16)
            e = cudaMemcpyAsync(r->host_out() + 4 * px, of + block_align(4 * px), 2 * px,
                                cudaMemcpyDeviceToHost, s.stream);
        if (e != cudaSuccess) st = cuda_fail(e, "server: result download");
    }
    if (st == VX_OK) {
        cudaError_t e = cudaEventRecord(s.done, s.stream);
        if (e != cudaSuccess) st = cuda_fail(e, "server: completion event");
    }
    s.reqs = batch;
    s.busy = true;
    if (st != VX_OK) {
        // Fail the whole batch; its block comes back once the stream drains.
        cudaStreamSynchronize(s.stream);
        cudaGetLastError();
        if (s.block_off != kNoBlock) dev_alloc.release(s.block_off, s.block_bytes);
        s.block_off = kNoBlock;
        std::lock_guard<std::mutex> lk(mu);
        for (Request* r : batch) {
            r->state = kFailed;
            r->status = st;
            r->t_done = Clock::now();
            ++stats.failed;
        }
        stats.inflight_bytes = dev_alloc.used();
        s.reqs.clear();
        s.busy = false;
        cv_done.notify_all();
    }
}

void vx_sgm_server::run() {
    DeviceGuard g(ctx->device);
    for (;;) {
        bool did = false;
        for (Slot& s : slots)
            if (s.busy && cudaEventQuery(s.done) == cudaSuccess) {
                retire(s);
                did = true;
            }
        cudaGetLastError();  // cudaErrorNotReady from the queries
        Slot* free_slot = nullptr;
        for (Slot& s : slots)
            if (!s.busy) {
                free_slot = &s;
                break;
            }
        std::vector<Request*> batch;
        {
            std::unique_lock<std::mutex> lk(mu);
            if (stop && pending.empty()) {
                bool any_busy = false;
                for (Slot& s : slots) any_busy |= s.busy;
                if (!any_busy) return;
            }
            if (free_slot) {
                // FIFO admission while the batch's bound fits one free block.
                const size_t room = dev_alloc.largest();
                size_t bytes = 0;
                while (!pending.empty() && batch.size() < max_batch) {
                    Request* r = pending.front();
                    if (r->state == kCancelled) {  // dropped while queued
                        pending.pop_front();
                        continue;
                    }
                    if (bytes + r->dev_bytes > room) break;  // wait for memory
                    pending.pop_front();
                    bytes += r->dev_bytes;
                    r->state = kRunning;
                    batch.push_back(r);
                }
                stats.queued = pending.size();
                if (!batch.empty()) ++stats.batches;
            }
            if (batch.empty() && !did) {
                bool any_busy = false;
                for (Slot& s : slots) any_busy |= s.busy;
                if (any_busy)
                    lk.unlock(), std::this_thread::sleep_for(std::chrono::microseconds(50));
                else
                    cv_work.wait_for(lk, std::chrono::milliseconds(5));
            }
        }
        if (!batch.empty()) {
            // Batches of other slots still running on the GPU when this one is
            // issued: their work and this batch's can overlap on the device.
            uint64_t in_flight = 1;
            for (Slot& o : slots)
                if (&o != free_slot && o.busy && cudaEventQuery(o.done) == cudaErrorNotReady) ++in_flight;
            cudaGetLastError();
            const auto t0 = Clock::now();
            launch(*free_slot, batch);
            const uint64_t us = (uint64_t)(ms_since(t0, Clock::now()) * 1e3);
            std::lock_guard<std::mutex> lk(mu);
            stats.max_launch_us = std::max(stats.max_launch_us, us);
            stats.max_batches_in_flight = std::max(stats.max_batches_in_flight, in_flight);
            stats.inflight_bytes = dev_alloc.used();
        }
    }
}

namespace {

void destroy_server(vx_sgm_server* s) {
    DeviceGuard g(s->ctx->device);
    for (auto& sl : s->slots) {
        if (sl.stream) {
            cudaStreamSynchronize(sl.stream);
            cudaStreamDestroy(sl.stream);
        }
        if (sl.done) cudaEventDestroy(sl.done);
        if (sl.esc_host) cudaFreeHost(sl.esc_host);
    }
    for (auto& kv : s->requests) s->host_put(kv.second.get());
    if (s->dev_arena) {
        cudaFreeAsync(s->dev_arena, s->ctx->stream);
        cudaStreamSynchronize(s->ctx->stream);
    }
    if (s->host_arena) cudaFreeHost(s->host_arena);
    cudaGetLastError();
    delete s;
}

}  // namespace

extern "C" {

vx_status vx_sgm_server_create(vx_sgm* sgm, vx_ctx* ctx, const vx_server_config* cfg,
                               vx_sgm_server** out) {
    if (!sgm || !ctx || !cfg || !out) return fail(VX_ERR_INVALID_ARGUMENT, "server_create: NULL argument");
    *out = nullptr;
    if (cfg->memory_budget_bytes < kBlockAlign || cfg->max_batch == 0 || cfg->max_inflight_batches == 0)
        return fail(VX_ERR_INVALID_CONFIG, "server_create: budget, max_batch and slots must be > 0");
    DeviceGuard g(ctx->device);
    auto* s = new vx_sgm_server;
    s->sgm = sgm;
    s->ctx = ctx;
    s->budget = cfg->memory_budget_bytes / kBlockAlign * kBlockAlign;
    s->max_batch = cfg->max_batch;
    s->slots.resize(cfg->max_inflight_batches);
    for (auto& sl : s->slots) {
        cudaError_t e = cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming);
        count_alloc();
        if (e == cudaSuccess)
            e = cudaMallocHost(reinterpret_cast<void**>(&sl.esc_host), 2 * sizeof(uint32_t) * cfg->max_batch);
        if (e != cudaSuccess) {
            vx_status st = cuda_fail(e, "server_create");
            destroy_server(s);
            return st;
        }
    }
    // The device arena: the whole budget, held for the server's lifetime.
    count_alloc();
    cudaError_t e = cudaMallocFromPoolAsync(reinterpret_cast<void**>(&s->dev_arena), s->budget, ctx->pool,
                                            ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        s->dev_arena = nullptr;
        destroy_server(s);
        return fail(VX_ERR_BUFFER_ALLOC, "server_create: device arena of %zu bytes", cfg->memory_budget_bytes);
    }
    s->dev_alloc.reset(s->budget);
    // The pinned staging arena (default: budget / 16, 256 MB .. 4 GB).
    size_t staging = cfg->host_staging_bytes;
    if (staging == 0) staging = std::min<size_t>(std::max<size_t>(s->budget / 16, 256u << 20), (size_t)4 << 30);
    staging = block_align(staging);
    count_alloc();
    if (cudaMallocHost(reinterpret_cast<void**>(&s->host_arena), staging) != cudaSuccess) {
        cudaGetLastError();
        s->host_arena = nullptr;
        destroy_server(s);
        return fail(VX_ERR_BUFFER_ALLOC, "server_create: pinned staging arena of %zu bytes", staging);
    }
    s->host_alloc.reset(staging);
    s->stats.pinned_bytes = staging;
    s->worker = std::thread([s] { s->run(); });
    *out = s;
    return VX_OK;
}

void vx_sgm_server_destroy(vx_sgm_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        for (Request* r : s->pending) {
            if (r->state == kPending) r->state = kCancelled;
        }
        s->pending.clear();
    }
    s->cv_work.notify_all();
    s->worker.join();
    destroy_server(s);
}

vx_status vx_sgm_server_submit(vx_sgm_server* s, const uint8_t* left, const uint8_t* right,
                               uint32_t width, uint32_t height, size_t host_pitch,
                               const vx_sgm_config* cfg, int want_i16, uint64_t* request_id) {
    if (!s || !left || !right || !cfg || !request_id)
        return fail(VX_ERR_INVALID_ARGUMENT, "server_submit: NULL argument");
    if (width == 0 || height == 0) return fail(VX_ERR_INVALID_ARGUMENT, "server_submit: empty image");
    if (host_pitch == 0) host_pitch = width;
    // Validate like a compute call (sizes, config) before queueing.
    vx_image l{nullptr, (void*)left, width, width, height, VX_FORMAT_U8, false};
    vx_image o{nullptr, (void*)left, (size_t)width * 4, width, height, VX_FORMAT_F32, false};
    vx_status st = validate_pair(PairSpec{&l, &l, &o, nullptr, *cfg});
    if (st != VX_OK) return st;
    auto r = std::make_unique<Request>();
    r->w = width;
    r->h = height;
    r->cfg = *cfg;
    r->want_i16 = want_i16 != 0;
    r->dev_bytes = vx_sgm_server::request_bytes(width, height, *cfg, r->want_i16, true);
    if (r->dev_bytes > s->budget) {
        std::lock_guard<std::mutex> lk(s->mu);
        ++s->stats.rejected;
        return fail(VX_ERR_BUDGET, "server_submit: request needs %zu device bytes, budget is %zu",
                    r->dev_bytes, s->budget);
    }
    if (!s->host_get(r.get())) return fail(VX_ERR_BUFFER_ALLOC, "server_submit: pinned host allocation failed");
    const size_t px = r->px();
    char* dst = r->host_in();
    for (uint32_t y = 0; y < height; ++y) {
        std::memcpy(dst + (size_t)y * width, left + (size_t)y * host_pitch, width);
        std::memcpy(dst + px + (size_t)y * width, right + (size_t)y * host_pitch, width);
    }
    r->t_submit = Clock::now();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stop) {
            s->host_put(r.get());
            return fail(VX_ERR_CANCELLED, "server_submit: server is shutting down");
        }
        r->id = s->next_id++;
        *request_id = r->id;
        s->pending.push_back(r.get());
        ++s->stats.submitted;
        s->stats.queued = s->pending.size();
        s->requests.emplace(r->id, std::move(r));
    }
    s->cv_work.notify_one();
    return VX_OK;
}

// Copies a finished request's result out and forgets it (caller holds mu).
static vx_status take_result(vx_sgm_server* s, Request* r, float* disparity, int16_t* disparity_i16,
                             double* latency_ms) {
    const size_t px = r->px();
    vx_status st = VX_OK;
    if (r->state == kDone) {
        if (disparity) std::memcpy(disparity, r->host_out(), 4 * px);
        if (disparity_i16 && r->want_i16) std::memcpy(disparity_i16, r->host_out() + 4 * px, 2 * px);
        if (latency_ms) *latency_ms = ms_since(r->t_submit, r->t_done);
    } else if (r->state == kCancelled) {
        st = fail(VX_ERR_CANCELLED, "request %llu was cancelled", (unsigned long long)r->id);
    } else {
        st = r->status != VX_OK ? r->status : VX_ERR_GPU;
    }
    s->host_put(r);
    s->requests.erase(r->id);
    return st;
}

vx_status vx_sgm_server_wait(vx_sgm_server* s, uint64_t id, float* disparity,
                             int16_t* disparity_i16, double* latency_ms, uint32_t timeout_ms) {
    if (!s) return fail(VX_ERR_INVALID_ARGUMENT, "server_wait: NULL server");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->requests.find(id);
    if (it == s->requests.end())
        return fail(VX_ERR_INVALID_ARGUMENT, "server_wait: unknown request %llu", (unsigned long long)id);
    Request* r = it->second.get();
    const auto pred = [&] { return r->state == kDone || r->state == kCancelled || r->state == kFailed; };
    if (timeout_ms == 0) {
        if (!pred()) return VX_ERR_NOT_READY;
    } else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), pred)) {
        return fail(VX_ERR_TIMEOUT, "server_wait: request %llu not done after %u ms",
                    (unsigned long long)id, timeout_ms);
    }
    return take_result(s, r, disparity, disparity_i16, latency_ms);
}

vx_status vx_sgm_server_cancel(vx_sgm_server* s, uint64_t id) {
    if (!s) return fail(VX_ERR_INVALID_ARGUMENT, "server_cancel: NULL server");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->requests.find(id);
    if (it == s->requests.end())
        return fail(VX_ERR_INVALID_ARGUMENT, "server_cancel: unknown request %llu", (unsigned long long)id);
    Request* r = it->second.get();
    if (r->state != kPending)
        return fail(VX_ERR_NOT_READY, "server_cancel: request %llu already started", (unsigned long long)id);
    r->state = kCancelled;
    s->pending.erase(std::find(s->pending.begin(), s->pending.end(), r));
    ++s->stats.cancelled;
    s->cv_done.notify_all();
    return VX_OK;
}

vx_status vx_sgm_server_get_stats(vx_sgm_server* s, vx_server_stats* out) {
    if (!s || !out) return fail(VX_ERR_INVALID_ARGUMENT, "server_get_stats: NULL argument");
    std::lock_guard<std::mutex> lk(s->mu);
    *out = s->stats;
    out->queued = s->pending.size();
    unsigned long long reserved = 0;
    if (cudaMemPoolGetAttribute(s->ctx->pool, cudaMemPoolAttrReservedMemCurrent, &reserved) != cudaSuccess)
        cudaGetLastError();
    out->pool_reserved_bytes = reserved;
    return VX_OK;
}

}  // extern "C"
