// StereoMatcher entry points of the vx_sgm C ABI (vx-vision/src/kernels/stereomatch.rs).
#include <cstdlib>
#include <cstring>
#include <mutex>

#include "vx_internal.hpp"

using namespace vxsgm;

static_assert(sizeof(vx_corner_point) == 16, "CornerPoint is 16 bytes (types.rs:8-12)");
static_assert(sizeof(vx_orb_output) == 36, "ORBOutput is 36 bytes (types.rs:36-39)");
static_assert(sizeof(vx_stereo_match_result) == 28, "StereoMatchResult is 28 bytes (types.rs:64-70)");
static_assert(sizeof(vx_stereo_match_result) == sizeof(StereoMatchRecord), "record layouts agree");

// The reference's StereoMatcher (stereomatch.rs:72-75) holds its two compiled
// pipelines. Here: the context, the matching scratch (keys, arrival counters,
// tile counts; grow-only) and, for the host-buffer entry point, a device block
// for inputs and results and a pinned host block that stages both directions.
struct vx_stereo_matcher {
    vx_ctx* ctx = nullptr;
    std::mutex mu;
    uint32_t* scratch = nullptr;  // keys[cap_left] | arrivals[cap_tiles] | tile_counts[cap_tiles]
    size_t cap_left = 0, cap_tiles = 0;
    bool scratch_dirty = false;  // a launch failed: the invariants of keys/arrivals are unknown
    // Banded form: bucket tables and sorted copies of cap_right right keypoints.
    char* band = nullptr;
    size_t band_cap_right = 0;
    bool band_dirty = false;
    char* dev_io = nullptr;
    size_t dev_io_bytes = 0;
    uint32_t* frame_offsets = nullptr;  // left | right offsets of the last frames call
    size_t frame_offsets_cap = 0;       // words
    char* host_io = nullptr;
    size_t host_io_bytes = 0;
};

namespace {

size_t round16(size_t v) { return (v + 15) & ~size_t(15); }

// Grows the matching scratch to n_left keys and its tiles; new or dirty scratch
// is reset on `stream` (keys to 0xFFFFFFFF, arrivals to 0).
vx_status ensure_scratch(vx_stereo_matcher* m, uint32_t n_left, const StereoMatchShape& shape,
                         cudaStream_t stream) {
    if (m->scratch && n_left <= m->cap_left && shape.left_tiles <= m->cap_tiles && !m->scratch_dirty)
        return VX_OK;
    size_t cap_left = m->cap_left, cap_tiles = m->cap_tiles;
    if (n_left > cap_left || shape.left_tiles > cap_tiles || !m->scratch) {
        cap_left = std::max<size_t>(n_left, cap_left * 2);
        // Tiles of 32 left keypoints (the banded form's) or of 256 (the other's).
        cap_tiles = std::max<size_t>(shape.left_tiles, (cap_left + 31) / 32);
        if (m->scratch) cudaFreeAsync(m->scratch, stream);
        m->scratch = nullptr;
        m->cap_left = m->cap_tiles = 0;
        count_alloc();
        cudaError_t e = cudaMallocFromPoolAsync(reinterpret_cast<void**>(&m->scratch),
                                                (cap_left + 2 * cap_tiles) * sizeof(uint32_t), m->ctx->pool, stream);
        if (e != cudaSuccess) return cuda_fail(e, "stereo matcher scratch");
        m->cap_left = cap_left;
        m->cap_tiles = cap_tiles;
    }
    cudaError_t e = cudaMemsetAsync(m->scratch, 0xFF, m->cap_left * sizeof(uint32_t), stream);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(m->scratch + m->cap_left, 0, 2 * m->cap_tiles * sizeof(uint32_t), stream);
    if (e != cudaSuccess) return cuda_fail(e, "stereo matcher scratch reset");
    m->scratch_dirty = false;
    return VX_OK;
}

// Bucket tables: hist[kRowBuckets+1] | arrival[1] | row_start[kRowBuckets+2] | cursor[kRowBuckets+1].
constexpr size_t kBandTableWords = 3 * (size_t)kRowBuckets + 5;
constexpr size_t kBandTableBytes = (kBandTableWords * 4 + 255) & ~size_t(255);

StereoBandScratch band_views(char* base, size_t cap_right) {
    StereoBandScratch b;
    uint32_t* t = reinterpret_cast<uint32_t*>(base);
    b.hist = t;
    b.arrival = t + kRowBuckets + 1;
    b.row_start = b.arrival + 1;
    b.cursor = b.row_start + kRowBuckets + 2;
    char* p = base + kBandTableBytes;
    b.desc = reinterpret_cast<uint4*>(p);
    p += 32 * cap_right;
    b.pos = reinterpret_cast<float2*>(p);
    p += 8 * cap_right;
    b.idx = reinterpret_cast<uint32_t*>(p);
    return b;
}

// Grows the banded form's scratch to n_right keypoints; new or dirty tables get
// hist and arrival cleared on `stream`.
vx_status ensure_band(vx_stereo_matcher* m, uint32_t n_right, cudaStream_t stream) {
    if (m->band && n_right <= m->band_cap_right && !m->band_dirty) return VX_OK;
    if (!m->band || n_right > m->band_cap_right) {
        const size_t cap = std::max<size_t>(n_right, m->band_cap_right * 2);
        if (m->band) cudaFreeAsync(m->band, stream);
        m->band = nullptr;
        m->band_cap_right = 0;
        count_alloc();
        cudaError_t e = cudaMallocFromPoolAsync(reinterpret_cast<void**>(&m->band), kBandTableBytes + 44 * cap,
                                                m->ctx->pool, stream);
        if (e != cudaSuccess) return cuda_fail(e, "stereo matcher band scratch");
        m->band_cap_right = cap;
    }
    cudaError_t e = cudaMemsetAsync(m->band, 0, (kRowBuckets + 2) * sizeof(uint32_t), stream);
    if (e != cudaSuccess) return cuda_fail(e, "stereo matcher band scratch reset");
    m->band_dirty = false;
    return VX_OK;
}

// The banded form pays two more launches and a scatter of the right keypoints
// and saves the pairs outside the epipolar band: it is used for 2^24 pairs and
// more (VX_STEREO_FORM=brute|banded forces one, where it applies).
bool use_banded(const vx_stereo_config* cfg, uint32_t n_left, uint32_t n_right) {
    const float e = cfg->max_epipolar;
    if (!(e >= 0.0f && e < kStereoBandMaxEpipolar)) return false;
    if (const char* f = std::getenv("VX_STEREO_FORM")) {
        if (!std::strcmp(f, "brute")) return false;
        if (!std::strcmp(f, "banded")) return true;
    }
    return (uint64_t)n_left * n_right >= (1ull << 24);
}

vx_status check_config(const vx_stereo_config* cfg) {
    if (!cfg) return fail(VX_ERR_INVALID_ARGUMENT, "stereo match: NULL config");
    return VX_OK;
}

StereoMatchParams make_params(const vx_stereo_config* cfg, uint32_t n_left, uint32_t n_right) {
    StereoMatchParams p{};
    p.n_left = n_left;
    p.n_right = n_right;
    p.max_epipolar = cfg->max_epipolar;
    p.min_disparity = cfg->min_disparity;
    p.max_disparity = cfg->max_disparity;
    p.max_hamming = cfg->max_hamming & 0xFFFFu;  // ushort(params.max_hamming), StereoMatch.metal:96
    p.fx = cfg->fx;
    p.fy = cfg->fy;
    p.cx = cfg->cx;
    p.cy = cfg->cy;
    p.baseline = cfg->baseline;
    return p;
}

// The device half shared by both entry points (m->mu held).
vx_status run_locked(vx_stereo_matcher* m, const vx_corner_point* lk, uint32_t n_left, const vx_corner_point* rk,
                     uint32_t n_right, const uint32_t* ld, const uint32_t* rd, const vx_stereo_config* cfg,
                     vx_stereo_match_result* out, uint32_t* count, cudaStream_t stream) {
    if (n_left == 0 || n_right == 0) {  // stereomatch.rs:138-142: no matches, no GPU work
        cudaError_t e = cudaMemsetAsync(count, 0, sizeof(uint32_t), stream);
        return e == cudaSuccess ? VX_OK : cuda_fail(e, "stereo match count");
    }
    const StereoMatchShape shape = stereo_match_shape(n_left, n_right, m->ctx->sm_count);
    vx_status st = ensure_scratch(m, n_left, shape, stream);
    if (st != VX_OK) return st;
    uint32_t* keys = m->scratch;
    uint32_t* arrivals = m->scratch + m->cap_left;
    uint32_t* tile_counts = arrivals + m->cap_tiles;
    if (use_banded(cfg, n_left, n_right)) {
        st = ensure_band(m, n_right, stream);
        if (st != VX_OK) return st;
        cudaError_t e = launch_stereo_match_banded(
            reinterpret_cast<const float4*>(lk), reinterpret_cast<const float4*>(rk),
            reinterpret_cast<const uint4*>(ld), reinterpret_cast<const uint4*>(rd), band_views(m->band, m->band_cap_right),
            keys, tile_counts, reinterpret_cast<StereoMatchRecord*>(out), count, make_params(cfg, n_left, n_right),
            m->ctx->sm_count, stream);
        if (e != cudaSuccess) {
            m->scratch_dirty = m->band_dirty = true;
            return cuda_fail(e, "stereo match launch");
        }
        return VX_OK;
    }
    cudaError_t e = launch_stereo_match(reinterpret_cast<const float4*>(lk), reinterpret_cast<const float4*>(rk),
                                        reinterpret_cast<const uint4*>(ld), reinterpret_cast<const uint4*>(rd),
                                        keys, arrivals, tile_counts, reinterpret_cast<StereoMatchRecord*>(out),
                                        count, make_params(cfg, n_left, n_right), shape, stream);
    if (e != cudaSuccess) {
        m->scratch_dirty = true;
        return cuda_fail(e, "stereo match launch");
    }
    return VX_OK;
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }
bool aligned4(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 3u) == 0; }

}  // namespace

extern "C" {

void vx_stereo_config_default(vx_stereo_config* cfg) {
    // StereoConfig::default (stereomatch.rs:54-69).
    if (cfg) *cfg = vx_stereo_config{2.0f, 1.0f, 120.0f, 50u, 0.8f, 600.0f, 600.0f, 320.0f, 240.0f, 0.12f};
}

vx_status vx_stereo_matcher_create(vx_ctx* ctx, vx_stereo_matcher** out) {
    if (!ctx || !out) return fail(VX_ERR_INVALID_ARGUMENT, "vx_stereo_matcher_create: NULL argument");
    auto* m = new vx_stereo_matcher;
    m->ctx = ctx;
    *out = m;
    return VX_OK;
}

void vx_stereo_matcher_destroy(vx_stereo_matcher* m) {
    if (!m) return;
    DeviceGuard g(m->ctx->device);
    cudaStreamSynchronize(m->ctx->stream);
    if (m->scratch) cudaFree(m->scratch);
    if (m->band) cudaFree(m->band);
    if (m->frame_offsets) cudaFree(m->frame_offsets);
    if (m->dev_io) cudaFree(m->dev_io);
    if (m->host_io) cudaFreeHost(m->host_io);
    delete m;
}

vx_status vx_stereo_matcher_run_device(vx_stereo_matcher* m, vx_ctx* ctx, const vx_corner_point* left_kpts,
                                       uint32_t n_left, const vx_corner_point* right_kpts, uint32_t n_right,
                                       const uint32_t* left_desc_words, const uint32_t* right_desc_words,
                                       const vx_stereo_config* cfg, vx_stereo_match_result* matches,
                                       uint32_t* match_count, vx_stream stream) {
    if (!m || !ctx || !match_count) return fail(VX_ERR_INVALID_ARGUMENT, "stereo match: NULL argument");
    vx_status st = check_config(cfg);
    if (st != VX_OK) return st;
    if (n_right > kStereoMaxRight || n_left > kStereoMaxLeft)
        return fail(VX_ERR_INVALID_ARGUMENT, "stereo match: at most %u left and %u right keypoints",
                    kStereoMaxLeft, kStereoMaxRight);
    if (n_left && n_right &&
        (!left_kpts || !right_kpts || !left_desc_words || !right_desc_words || !matches))
        return fail(VX_ERR_INVALID_ARGUMENT, "stereo match: NULL device pointer");
    if (!aligned16(left_kpts) || !aligned16(right_kpts) || !aligned16(left_desc_words) ||
        !aligned16(right_desc_words) || !aligned4(matches) || !aligned4(match_count))
        return fail(VX_ERR_INVALID_ARGUMENT,
                    "stereo match: keypoints and descriptors must be 16-byte aligned, results 4-byte aligned");
    DeviceGuard g(ctx->device);
    cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
    std::lock_guard<std::mutex> lock(m->mu);
    st = run_locked(m, left_kpts, n_left, right_kpts, n_right, left_desc_words, right_desc_words, cfg, matches,
                    match_count, s);
    if (st != VX_OK) return st;
    if (!stream) {
        cudaError_t e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return cuda_fail(e, "stereo match");
    }
    return VX_OK;
}

vx_status vx_stereo_matcher_run_frames_device(vx_stereo_matcher* m, vx_ctx* ctx, uint32_t n_frames,
                                              const uint32_t* left_offsets, const uint32_t* right_offsets,
                                              const vx_corner_point* left_kpts, const vx_corner_point* right_kpts,
                                              const uint32_t* left_desc_words, const uint32_t* right_desc_words,
                                              const vx_stereo_config* cfg, vx_stereo_match_result* matches,
                                              uint32_t* match_counts, vx_stream stream) {
    if (!m || !ctx || !left_offsets || !right_offsets || !match_counts)
        return fail(VX_ERR_INVALID_ARGUMENT, "stereo frames: NULL argument");
    vx_status st = check_config(cfg);
    if (st != VX_OK) return st;
    if (n_frames == 0) return VX_OK;
    if (left_offsets[0] != 0 || right_offsets[0] != 0)
        return fail(VX_ERR_INVALID_ARGUMENT, "stereo frames: offsets must start at 0");
    for (uint32_t f = 0; f < n_frames; ++f) {
        if (left_offsets[f + 1] < left_offsets[f] || right_offsets[f + 1] < right_offsets[f])
            return fail(VX_ERR_INVALID_ARGUMENT, "stereo frames: offsets of frame %u decrease", f);
        if (right_offsets[f + 1] - right_offsets[f] > kStereoMaxRight)
            return fail(VX_ERR_INVALID_ARGUMENT, "stereo frames: frame %u has more than %u right keypoints", f,
                        kStereoMaxRight);
    }
    const uint32_t nl = left_offsets[n_frames], nr = right_offsets[n_frames];
    if ((nl && (!left_kpts || !left_desc_words || !matches)) || (nr && (!right_kpts || !right_desc_words)))
        return fail(VX_ERR_INVALID_ARGUMENT, "stereo frames: NULL device pointer");
    if (!aligned16(left_kpts) || !aligned16(right_kpts) || !aligned16(left_desc_words) ||
        !aligned16(right_desc_words) || !aligned4(matches) || !aligned4(match_counts))
        return fail(VX_ERR_INVALID_ARGUMENT,
                    "stereo frames: keypoints and descriptors must be 16-byte aligned, results 4-byte aligned");
    DeviceGuard g(ctx->device);
    cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
    std::lock_guard<std::mutex> lock(m->mu);
    const size_t words = 2 * ((size_t)n_frames + 1);
    if (m->frame_offsets_cap < words) {
        const size_t cap = std::max(words, 2 * m->frame_offsets_cap);
        if (m->frame_offsets) cudaFreeAsync(m->frame_offsets, s);
        m->frame_offsets = nullptr;
        m->frame_offsets_cap = 0;
        count_alloc();
        cudaError_t e = cudaMallocFromPoolAsync(reinterpret_cast<void**>(&m->frame_offsets), cap * sizeof(uint32_t),
                                                ctx->pool, s);
        if (e != cudaSuccess) return cuda_fail(e, "stereo frames offsets");
        m->frame_offsets_cap = cap;
    }
    // Pageable sources: the copies are staged before they return.
    cudaError_t e = cudaMemcpyAsync(m->frame_offsets, left_offsets, (n_frames + 1) * sizeof(uint32_t),
                                    cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(m->frame_offsets + n_frames + 1, right_offsets, (n_frames + 1) * sizeof(uint32_t),
                            cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = launch_stereo_match_frames(reinterpret_cast<const float4*>(left_kpts),
                                       reinterpret_cast<const float4*>(right_kpts),
                                       reinterpret_cast<const uint4*>(left_desc_words),
                                       reinterpret_cast<const uint4*>(right_desc_words), m->frame_offsets,
                                       m->frame_offsets + n_frames + 1, n_frames,
                                       reinterpret_cast<StereoMatchRecord*>(matches), match_counts,
                                       make_params(cfg, 0, 0), s);
    if (e == cudaSuccess && !stream) e = cudaStreamSynchronize(s);
    return e == cudaSuccess ? VX_OK : cuda_fail(e, "stereo frames");
}

vx_status vx_stereo_matcher_run(vx_stereo_matcher* m, vx_ctx* ctx, const vx_corner_point* left_kpts,
                                size_t n_left_kpts, const vx_corner_point* right_kpts, size_t n_right_kpts,
                                const vx_orb_output* left_descs, size_t n_left_descs, const vx_orb_output* right_descs,
                                size_t n_right_descs, const vx_stereo_config* cfg, vx_stereo_match_result* matches,
                                size_t capacity, size_t* n_matches) {
    if (!m || !ctx || !n_matches) return fail(VX_ERR_INVALID_ARGUMENT, "stereo match: NULL argument");
    *n_matches = 0;
    vx_status st = check_config(cfg);
    if (st != VX_OK) return st;
    // stereomatch.rs:124-133 asserts these; a C caller gets an error instead.
    if (n_left_kpts != n_left_descs)
        return fail(VX_ERR_INVALID_ARGUMENT, "left_kpts and left_descs length mismatch (%zu vs %zu)", n_left_kpts,
                    n_left_descs);
    if (n_right_kpts != n_right_descs)
        return fail(VX_ERR_INVALID_ARGUMENT, "right_kpts and right_descs length mismatch (%zu vs %zu)",
                    n_right_kpts, n_right_descs);
    if (n_right_kpts > kStereoMaxRight || n_left_kpts > kStereoMaxLeft)
        return fail(VX_ERR_INVALID_ARGUMENT, "stereo match: at most %u left and %u right keypoints",
                    kStereoMaxLeft, kStereoMaxRight);
    const uint32_t nl = (uint32_t)n_left_kpts, nr = (uint32_t)n_right_kpts;
    if (nl == 0 || nr == 0) return VX_OK;  // stereomatch.rs:138-142
    if (!left_kpts || !right_kpts || !left_descs || !right_descs || !matches)
        return fail(VX_ERR_INVALID_ARGUMENT, "stereo match: NULL buffer");
    if (capacity < nl)
        return fail(VX_ERR_INVALID_ARGUMENT, "stereo match: room for %zu matches, up to %u possible", capacity, nl);

    // One staging layout for both directions: inputs | count (16 bytes) | records.
    const size_t off_rk = round16(16ull * nl), off_ld = off_rk + round16(16ull * nr);
    const size_t off_rd = off_ld + 32ull * nl, in_bytes = round16(off_rd + 32ull * nr);
    const size_t out_bytes = 16 + sizeof(vx_stereo_match_result) * (size_t)nl;
    const size_t total = in_bytes + round16(out_bytes);

    DeviceGuard g(ctx->device);
    cudaStream_t s = ctx->stream;
    std::lock_guard<std::mutex> lock(m->mu);
    if (m->host_io_bytes < total) {
        if (m->host_io) {
            cudaStreamSynchronize(s);
            cudaFreeHost(m->host_io);
        }
        m->host_io = nullptr;
        m->host_io_bytes = 0;
        count_alloc();
        if (cudaMallocHost(reinterpret_cast<void**>(&m->host_io), total) != cudaSuccess)
            return fail(VX_ERR_BUFFER_ALLOC, "stereo match: %zu bytes of pinned staging", total);
        m->host_io_bytes = total;
    }
    if (m->dev_io_bytes < total) {
        if (m->dev_io) cudaFreeAsync(m->dev_io, s);
        m->dev_io = nullptr;
        m->dev_io_bytes = 0;
        count_alloc();
        cudaError_t e = cudaMallocFromPoolAsync(reinterpret_cast<void**>(&m->dev_io), total, ctx->pool, s);
        if (e != cudaSuccess) return cuda_fail(e, "stereo match device staging");
        m->dev_io_bytes = total;
    }
    // The reference's host side flattens the descriptors to 8 words per
    // keypoint (stereomatch.rs:144-145); here while filling the pinned block.
    char* h = m->host_io;
    std::memcpy(h, left_kpts, 16ull * nl);
    std::memcpy(h + off_rk, right_kpts, 16ull * nr);
    uint32_t* hld = reinterpret_cast<uint32_t*>(h + off_ld);
    for (uint32_t i = 0; i < nl; ++i) std::memcpy(hld + 8ull * i, left_descs[i].desc, 32);
    uint32_t* hrd = reinterpret_cast<uint32_t*>(h + off_rd);
    for (uint32_t i = 0; i < nr; ++i) std::memcpy(hrd + 8ull * i, right_descs[i].desc, 32);

    char* d = m->dev_io;
    cudaError_t e = cudaMemcpyAsync(d, h, off_rd + 32ull * nr, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return cuda_fail(e, "stereo match upload");
    uint32_t* d_count = reinterpret_cast<uint32_t*>(d + in_bytes);
    auto* d_out = reinterpret_cast<vx_stereo_match_result*>(d + in_bytes + 16);
    st = run_locked(m, reinterpret_cast<const vx_corner_point*>(d), nl,
                    reinterpret_cast<const vx_corner_point*>(d + off_rk), nr,
                    reinterpret_cast<const uint32_t*>(d + off_ld), reinterpret_cast<const uint32_t*>(d + off_rd), cfg,
                    d_out, d_count, s);
    if (st != VX_OK) return st;
    e = cudaMemcpyAsync(h + in_bytes, d + in_bytes, out_bytes, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(e, "stereo match");
    uint32_t n = 0;
    std::memcpy(&n, h + in_bytes, sizeof(n));
    if (n > nl) n = nl;  // stereomatch.rs:245
    std::memcpy(matches, h + in_bytes + 16, sizeof(vx_stereo_match_result) * (size_t)n);
    *n_matches = n;
    return VX_OK;
}

}  // extern "C"
