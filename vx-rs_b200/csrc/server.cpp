// Serving loop: continuous batching of stereo requests under a device-memory
// budget (no counterpart in vx-vision, whose SGM call is one synchronous pair,
// vx-vision/src/kernels/sgm.rs:108-265).
//
// Requests are submitted from any host thread; their images are copied into
// pinned host buffers from a reuse pool. A scheduler thread
//  * retires batches whose completion event has fired (results are already in
//    the request's pinned output buffer; device memory goes back to the
//    context's pool and to the budget),
//  * admits pending requests in arrival order while their device bytes
//    (workspace + images + outputs) fit the remaining budget, up to max_batch
//    per batch, as soon as one of max_inflight stream slots is free, and
//  * launches the batch on that slot's stream: H2D of the images, the batched
//    SGM (census, one persistent aggregation launch, WTA), D2H of the
//    disparities, completion event.
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

// Pinned host buffers by power-of-two size class, reused across requests.
// cudaMallocHost is slow and serialises with other CUDA calls, so blocks are
// carved out of chunks of at least 64 MB (and 8 blocks) per class.
class PinnedPool {
  public:
    ~PinnedPool() {
        for (void* c : chunks_) cudaFreeHost(c);
    }
    void* get(size_t bytes, size_t* cls) {
        size_t c = 4096;
        while (c < bytes) c <<= 1;
        *cls = c;
        std::lock_guard<std::mutex> lk(mu_);
        auto& v = free_[c];
        if (v.empty()) {
            const size_t n = std::max<size_t>(8, ((size_t)64 << 20) / c);
            void* chunk = nullptr;
            if (cudaMallocHost(&chunk, n * c) != cudaSuccess) {
                cudaGetLastError();
                return nullptr;
            }
            chunks_.push_back(chunk);
            for (size_t i = 0; i < n; ++i) v.push_back(static_cast<char*>(chunk) + i * c);
        }
        void* p = v.back();
        v.pop_back();
        return p;
    }
    void put(void* p, size_t cls) {
        if (!p) return;
        std::lock_guard<std::mutex> lk(mu_);
        free_[cls].push_back(p);
    }

  private:
    std::mutex mu_;
    std::map<size_t, std::vector<void*>> free_;
    std::vector<void*> chunks_;
};

enum ReqState { kPending, kRunning, kDone, kCancelled, kFailed };

struct Request {
    uint64_t id = 0;
    uint32_t w = 0, h = 0;
    vx_sgm_config cfg{};
    bool want_i16 = false;
    void* host_in = nullptr;   // left then right, w*h each
    size_t in_cls = 0;
    void* host_out = nullptr;  // f32 disparity (w*h), then i16 (w*h) if wanted
    size_t out_cls = 0;
    size_t dev_bytes = 0;      // charged against the budget while running
    void* dev_buf = nullptr;   // images + outputs on the device
    Clock::time_point t_submit, t_done;
    ReqState state = kPending;
    vx_status status = VX_OK;
};

struct Slot {
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    std::vector<Request*> reqs;
    bool busy = false;
};

}  // namespace
}  // namespace vxsgm

using namespace vxsgm;

struct vx_sgm_server {
    vx_sgm* sgm = nullptr;
    vx_ctx* ctx = nullptr;
    size_t budget = 0;
    uint32_t max_batch = 0;
    std::vector<Slot> slots;
    PinnedPool pinned;

    std::mutex mu;
    std::condition_variable cv_work;  // new submissions / stop
    std::condition_variable cv_done;  // a request finished
    std::deque<Request*> pending;
    std::unordered_map<uint64_t, std::unique_ptr<Request>> requests;
    uint64_t next_id = 1;
    size_t inflight_bytes = 0;
    bool stop = false;
    vx_server_stats stats{};
    std::thread worker;

    size_t request_bytes(uint32_t w, uint32_t h, const vx_sgm_config& cfg, bool i16) const {
        const size_t px = (size_t)w * h;
        return vx_sgm_workspace_bytes(w, h, &cfg) + 2 * px + 4 * px + (i16 ? 2 * px : 0) + 4096;
    }

    void run();
    void retire(Slot& s);
    void launch(Slot& s, std::vector<Request*>& batch);
};

void vx_sgm_server::retire(Slot& s) {
    const auto now = Clock::now();
    for (Request* r : s.reqs) {
        cudaFreeAsync(r->dev_buf, s.stream);
        r->dev_buf = nullptr;
    }
    std::lock_guard<std::mutex> lk(mu);
    for (Request* r : s.reqs) {
        inflight_bytes -= r->dev_bytes;
        r->t_done = now;
        if (r->state == kRunning) {
            r->state = kDone;
            ++stats.completed;
            stats.completed_pixel_disparities +=
                (uint64_t)r->w * r->h * r->cfg.num_disparities;
        }
    }
    stats.inflight_bytes = inflight_bytes;
    s.reqs.clear();
    s.busy = false;
    cv_done.notify_all();
}

void vx_sgm_server::launch(Slot& s, std::vector<Request*>& batch) {
    DeviceGuard g(ctx->device);
    std::vector<vx_image> imgs(batch.size() * 4);
    std::vector<PairSpec> specs;
    vx_status st = VX_OK;
    for (size_t i = 0; i < batch.size() && st == VX_OK; ++i) {
        Request* r = batch[i];
        const size_t px = (size_t)r->w * r->h;
        const size_t bytes = 2 * px + 4 * px + (r->want_i16 ? 2 * px : 0) + 256;
        cudaError_t e = cudaMallocFromPoolAsync(&r->dev_buf, bytes, ctx->pool, s.stream);
        if (e != cudaSuccess) {
            cudaGetLastError();
            st = fail(VX_ERR_BUFFER_ALLOC, "server: buffer allocation failed (%zu bytes)", bytes);
            break;
        }
        char* base = static_cast<char*>(r->dev_buf);
        // f32 output first (4-byte aligned), then i16, then the two u8 images.
        char* of = base;
        char* oi = base + 4 * px;
        char* li = oi + (r->want_i16 ? 2 * px : 0);
        char* ri = li + px;
        e = cudaMemcpyAsync(li, r->host_in, 2 * px, cudaMemcpyHostToDevice, s.stream);
        if (e != cudaSuccess) st = cuda_fail(e, "server: image upload");
        vx_image* im = &imgs[4 * i];
        im[0] = {ctx, li, r->w, r->w, r->h, VX_FORMAT_U8, false};
        im[1] = {ctx, ri, r->w, r->w, r->h, VX_FORMAT_U8, false};
        im[2] = {ctx, of, (size_t)r->w * 4, r->w, r->h, VX_FORMAT_F32, false};
        im[3] = {ctx, oi, (size_t)r->w * 2, r->w, r->h, VX_FORMAT_I16, false};
        specs.push_back({&im[0], &im[1], &im[2], r->want_i16 ? &im[3] : nullptr, r->cfg});
    }
    if (st == VX_OK) st = run_batch_plain(sgm, ctx, specs, s.stream);
    for (size_t i = 0; i < batch.size() && st == VX_OK; ++i) {
        Request* r = batch[i];
        const size_t px = (size_t)r->w * r->h;
        const size_t out = 4 * px + (r->want_i16 ? 2 * px : 0);
        cudaError_t e = cudaMemcpyAsync(r->host_out, r->dev_buf, out, cudaMemcpyDeviceToHost, s.stream);
        if (e != cudaSuccess) st = cuda_fail(e, "server: result download");
    }
    if (st == VX_OK) {
        cudaError_t e = cudaEventRecord(s.done, s.stream);
        if (e != cudaSuccess) st = cuda_fail(e, "server: completion event");
    }
    s.reqs = batch;
    s.busy = true;
    if (st != VX_OK) {
        // Fail the whole batch; its memory comes back when the stream drains.
        cudaStreamSynchronize(s.stream);
        std::lock_guard<std::mutex> lk(mu);
        for (Request* r : batch) {
            r->state = kFailed;
            r->status = st;
            ++stats.failed;
        }
        for (Request* r : batch) {
            if (r->dev_buf) cudaFreeAsync(r->dev_buf, s.stream);
            r->dev_buf = nullptr;
            inflight_bytes -= r->dev_bytes;
            r->t_done = Clock::now();
        }
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
                while (!pending.empty() && batch.size() < max_batch) {
                    Request* r = pending.front();
                    if (r->state == kCancelled) {  // dropped while queued
                        pending.pop_front();
                        continue;
                    }
                    if (inflight_bytes + r->dev_bytes > budget) break;  // FIFO: wait for memory
                    pending.pop_front();
                    inflight_bytes += r->dev_bytes;
                    r->state = kRunning;
                    batch.push_back(r);
                }
                stats.inflight_bytes = inflight_bytes;
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
        if (!batch.empty()) launch(*free_slot, batch);
    }
}

extern "C" {

vx_status vx_sgm_server_create(vx_sgm* sgm, vx_ctx* ctx, const vx_server_config* cfg,
                               vx_sgm_server** out) {
    if (!sgm || !ctx || !cfg || !out) return fail(VX_ERR_INVALID_ARGUMENT, "server_create: NULL argument");
    *out = nullptr;
    if (cfg->memory_budget_bytes == 0 || cfg->max_batch == 0 || cfg->max_inflight_batches == 0)
        return fail(VX_ERR_INVALID_CONFIG, "server_create: budget, max_batch and slots must be > 0");
    DeviceGuard g(ctx->device);
    auto* s = new vx_sgm_server;
    s->sgm = sgm;
    s->ctx = ctx;
    s->budget = cfg->memory_budget_bytes;
    s->max_batch = cfg->max_batch;
    s->slots.resize(cfg->max_inflight_batches);
    for (auto& sl : s->slots) {
        cudaError_t e = cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming);
        if (e != cudaSuccess) {
            vx_status st = cuda_fail(e, "server_create");
            for (auto& x : s->slots) {
                if (x.stream) cudaStreamDestroy(x.stream);
                if (x.done) cudaEventDestroy(x.done);
            }
            delete s;
            return st;
        }
    }
    // Keep the budget resident: map it into the context's pool now, so that
    // admitting requests never waits for the pool to grow.
    {
        void* warm = nullptr;
        if (cudaMallocFromPoolAsync(&warm, s->budget, ctx->pool, s->slots[0].stream) == cudaSuccess) {
            cudaFreeAsync(warm, s->slots[0].stream);
            cudaStreamSynchronize(s->slots[0].stream);
        } else {
            cudaGetLastError();  // the pool grows on demand instead
        }
    }
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
    DeviceGuard g(s->ctx->device);
    for (auto& sl : s->slots) {
        cudaStreamSynchronize(sl.stream);
        cudaStreamDestroy(sl.stream);
        cudaEventDestroy(sl.done);
    }
    for (auto& kv : s->requests) {
        s->pinned.put(kv.second->host_in, kv.second->in_cls);
        s->pinned.put(kv.second->host_out, kv.second->out_cls);
    }
    delete s;
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
    r->dev_bytes = s->request_bytes(width, height, *cfg, r->want_i16);
    if (r->dev_bytes > s->budget) {
        std::lock_guard<std::mutex> lk(s->mu);
        ++s->stats.rejected;
        return fail(VX_ERR_BUDGET, "server_submit: request needs %zu device bytes, budget is %zu",
                    r->dev_bytes, s->budget);
    }
    const size_t px = (size_t)width * height;
    r->host_in = s->pinned.get(2 * px, &r->in_cls);
    r->host_out = s->pinned.get(4 * px + (r->want_i16 ? 2 * px : 0), &r->out_cls);
    if (!r->host_in || !r->host_out) {
        s->pinned.put(r->host_in, r->in_cls);
        s->pinned.put(r->host_out, r->out_cls);
        return fail(VX_ERR_BUFFER_ALLOC, "server_submit: pinned host allocation failed");
    }
    uint8_t* dst = static_cast<uint8_t*>(r->host_in);
    for (uint32_t y = 0; y < height; ++y) {
        std::memcpy(dst + (size_t)y * width, left + (size_t)y * host_pitch, width);
        std::memcpy(dst + px + (size_t)y * width, right + (size_t)y * host_pitch, width);
    }
    r->t_submit = Clock::now();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stop) return fail(VX_ERR_CANCELLED, "server_submit: server is shutting down");
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

// Copies a finished request's result out and forgets it.
static vx_status take_result(vx_sgm_server* s, std::unique_lock<std::mutex>& lk, Request* r,
                             float* disparity, int16_t* disparity_i16, double* latency_ms) {
    (void)lk;
    const size_t px = (size_t)r->w * r->h;
    vx_status st = VX_OK;
    if (r->state == kDone) {
        if (disparity) std::memcpy(disparity, r->host_out, 4 * px);
        if (disparity_i16 && r->want_i16)
            std::memcpy(disparity_i16, static_cast<char*>(r->host_out) + 4 * px, 2 * px);
        if (latency_ms) *latency_ms = ms_since(r->t_submit, r->t_done);
    } else if (r->state == kCancelled) {
        st = fail(VX_ERR_CANCELLED, "request %llu was cancelled", (unsigned long long)r->id);
    } else {
        st = r->status != VX_OK ? r->status : VX_ERR_GPU;
    }
    s->pinned.put(r->host_in, r->in_cls);
    s->pinned.put(r->host_out, r->out_cls);
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
    return take_result(s, lk, r, disparity, disparity_i16, latency_ms);
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
    out->inflight_bytes = s->inflight_bytes;
    return VX_OK;
}

}  // extern "C"
