/*
 * vx_sgm.h - C ABI of the B200 (sm_100a) semi-global matching stereo library.
 *
 * Drop-in boundary for vx-vision's SGM path (MisterEkole/vx-rs). Each entry
 * point names the reference interface it replaces (paths are within the
 * vx-rs project). Plain C types only: pointers, sizes, enums, PODs.
 *
 * Semantics follow vx-vision/shaders/SGMStereo.metal exactly (census, Hamming
 * cost with 64 for x-d < 0, the shader's in-place u16 path recurrence, u16
 * accumulation, first-minimum WTA, parabola subpixel). Extensions over the
 * reference are opt-in config fields: 4/8 paths and a left-right check.
 *
 * Threading: every handle may be shared between host threads; calls that
 * take a stream are ordered on that stream, calls given a NULL stream are
 * synchronous like the reference's commit() + waitUntilCompleted()
 * (vx-vision/src/kernels/sgm.rs:260-261).
 */
#ifndef VX_SGM_H
#define VX_SGM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Mirrors vx-vision/src/error.rs:8-23 (Error), plus codes for the additions. */
typedef enum vx_status {
    VX_OK = 0,
    VX_ERR_DEVICE_NOT_FOUND = 1,   /* Error::DeviceNotFound */
    VX_ERR_SHADER_MISSING = 2,     /* Error::ShaderMissing: kernel image absent for this GPU */
    VX_ERR_PIPELINE_COMPILE = 3,   /* Error::PipelineCompile */
    VX_ERR_BUFFER_ALLOC = 4,       /* Error::BufferAlloc { bytes } */
    VX_ERR_SIZE_MISMATCH = 5,      /* Error::TextureSizeMismatch */
    VX_ERR_INVALID_CONFIG = 6,     /* Error::InvalidConfig(String) */
    VX_ERR_GPU = 7,                /* Error::Gpu(String) */
    VX_ERR_BUDGET = 8,             /* request larger than the server's memory budget */
    VX_ERR_TIMEOUT = 9,            /* a bounded wait gave up */
    VX_ERR_INVALID_ARGUMENT = 10,  /* null handle / pointer, bad format */
    VX_ERR_NOT_READY = 11,         /* asynchronous result not finished yet */
    VX_ERR_CANCELLED = 12          /* request cancelled before it ran */
} vx_status;

/* Human-readable detail of the last error on the calling host thread
 * (the String payloads of vx-vision's Error). Never NULL. */
const char* vx_last_error(void);

typedef struct vx_ctx vx_ctx;
typedef struct vx_image vx_image;
typedef struct vx_sgm vx_sgm;
typedef void* vx_stream; /* a cudaStream_t; NULL = synchronous call */

/* Replaces Context::new() (vx-vision/src/context.rs:26): selects a CUDA
 * device, creates its stream and a stream-ordered device memory pool. */
vx_status vx_ctx_create(int device_ordinal, vx_ctx** out);
void vx_ctx_destroy(vx_ctx* ctx);
/* The context's default stream (Context::queue(), context.rs:83). */
vx_stream vx_ctx_stream(vx_ctx* ctx);
/* Blocks until all work on the context's stream has finished. */
vx_status vx_ctx_synchronize(vx_ctx* ctx);
/* Largest device workspace one batch call may take (default: 85% of the device
 * memory free when the context was created). A batch needing more runs as
 * consecutive sub-batches on the same stream. */
vx_status vx_ctx_set_workspace_limit(vx_ctx* ctx, size_t bytes);

/* Image formats: R8Unorm input (texture.rs:38 from_gray8), R32Float output
 * (texture.rs:324 output_r32float), an int16 integer-disparity map, and
 * RGBA8Unorm colour images (Context::texture_rgba8, context.rs:54; bytes r, g,
 * b, a per pixel). */
typedef enum vx_format { VX_FORMAT_U8 = 0, VX_FORMAT_F32 = 1, VX_FORMAT_I16 = 2, VX_FORMAT_RGBA8 = 3 } vx_format;

/* Replaces Context::texture_gray8 / texture_output_r32float
 * (context.rs:39, context.rs:64): allocates a pitched device image. */
vx_status vx_image_create(vx_ctx* ctx, uint32_t width, uint32_t height, vx_format format,
                          vx_image** out);
/* Replaces Texture::from_metal_texture (texture.rs:449): wraps caller-owned
 * device memory (pitch in bytes). The image never frees it. */
vx_status vx_image_wrap_device(vx_ctx* ctx, void* device_ptr, size_t pitch_bytes, uint32_t width,
                               uint32_t height, vx_format format, vx_image** out);
void vx_image_destroy(vx_image* img);
uint32_t vx_image_width(const vx_image* img);   /* Texture::width, texture.rs */
uint32_t vx_image_height(const vx_image* img);  /* Texture::height */
void* vx_image_device_ptr(const vx_image* img);
size_t vx_image_pitch(const vx_image* img);
/* Host <-> device copies. Replace Texture::from_gray8's replaceRegion
 * (texture.rs:38-75) and Texture::read_r32float (texture.rs:404).
 * host_pitch in bytes (0 = tightly packed). NULL stream = synchronous. */
vx_status vx_image_upload(vx_image* img, const void* host, size_t host_pitch, vx_stream stream);
vx_status vx_image_download(const vx_image* img, void* host, size_t host_pitch, vx_stream stream);

/* Replaces SGMStereoConfig (vx-vision/src/kernels/sgm.rs:23-37). The first
 * five fields are the reference's; the rest are extensions whose defaults
 * reproduce the reference (2 paths, subpixel on, no LR check). */
typedef struct vx_sgm_config {
    uint32_t num_disparities; /* 1..256 (SGMStereo.metal:108 caps at 256) */
    float p1;                 /* penalty for |dd| = 1, used as ushort(p1) */
    float p2;                 /* penalty for |dd| > 1, used as ushort(p2) */
    uint32_t census_radius_x;
    uint32_t census_radius_y; /* (2rx+1)(2ry+1)-1 <= 64 census bits */
    uint32_t num_paths;       /* 2 = reference ((1,0),(0,1)); 4; 8 */
    uint32_t subpixel;        /* 1 = parabola refinement (reference) */
    uint32_t lr_check;        /* 1 = left-right consistency check */
    uint32_t lr_tolerance;    /* pixels */
    float invalid_value;      /* written where the LR check fails */
} vx_sgm_config;

/* SGMStereoConfig::default() (sgm.rs:39-49): D=128, P1=10, P2=120, 4x3. */
void vx_sgm_config_default(vx_sgm_config* cfg);
/* SGMStereoConfig::new(num_disparities) (sgm.rs:51-59). */
void vx_sgm_config_new(vx_sgm_config* cfg, uint32_t num_disparities);

/* Replaces SGMStereo::new(&ctx) (sgm.rs:73-105): checks that the sm_100a
 * kernel images load on the context's device (ShaderMissing otherwise). */
vx_status vx_sgm_create(vx_ctx* ctx, vx_sgm** out);
void vx_sgm_destroy(vx_sgm* sgm);  /* before the context it was created with */

/* Replaces SGMStereo::compute_disparity(&ctx, &left, &right, &output, &cfg)
 * (sgm.rs:108-265). left/right: U8 images of equal size; out_f32: F32 image
 * of that size (subpixel disparity, or invalid_value); out_i16: optional I16
 * image (integer disparity, -1 where invalid). Unlike the reference, sizes and
 * config are validated (VX_ERR_SIZE_MISMATCH / VX_ERR_INVALID_CONFIG).
 * Intermediates come from the context's stream-ordered pool. */
vx_status vx_sgm_compute_disparity(vx_sgm* sgm, vx_ctx* ctx, const vx_image* left,
                                   const vx_image* right, vx_image* out_f32, vx_image* out_i16,
                                   const vx_sgm_config* cfg, vx_stream stream);

/* CameraIntrinsics (vx-vision/src/types_3d.rs:254-267). */
typedef struct vx_camera_intrinsics {
    float fx, fy, cx, cy;
    uint32_t width, height;
} vx_camera_intrinsics;

/* DepthMap (vx-vision/src/types_3d.rs:384-410): an F32 texture with intrinsics
 * and a depth range. The texture is owned by the caller (vx_image_destroy). */
typedef struct vx_depth_map {
    vx_image* texture;
    vx_camera_intrinsics intrinsics;
    float min_depth, max_depth;
} vx_depth_map;

/* Replaces SGMStereo::compute(&ctx, &left, &right, &config, &intrinsics,
 * baseline) (sgm.rs:268-288): allocates an F32 output of the left image's size,
 * computes the disparity into it and returns a DepthMap over it with
 * min_depth 0 and max_depth FLT_MAX, exactly like the reference (which does
 * not convert disparity to depth and ignores baseline). Extension: if depth_out
 * (an F32 image of the same size) is given, the WTA kernel also writes
 * depth = fx * baseline / disparity there (0 where the disparity is invalid or
 * <= 0). Synchronous on the context's stream. */
vx_status vx_sgm_compute(vx_sgm* sgm, vx_ctx* ctx, const vx_image* left, const vx_image* right,
                         const vx_sgm_config* cfg, const vx_camera_intrinsics* intrinsics,
                         float baseline, vx_image* depth_out, vx_depth_map* out);

/* Batched form of compute_disparity (no reference counterpart; the
 * reference only has the per-pair call, sgm.rs:108): n independent pairs of
 * any sizes and configs in one pass: one census launch, path aggregation as
 * persistent launches over a (pair, path, scanline-group) work queue, one
 * WTA launch. out_i16 may be NULL or contain NULLs. A synchronous call (NULL
 * stream, graph cache off) keeps each pair's rare escaped path vectors (values
 * above a byte) in a pool of 1/16 of its vectors instead of a full u16 shadow,
 * about a third of the workspace, and recomputes any pair whose pool ran out
 * with a full shadow, so results are the same either way. */
vx_status vx_sgm_compute_batch(vx_sgm* sgm, vx_ctx* ctx, uint32_t n, const vx_image* const* left,
                               const vx_image* const* right, vx_image* const* out_f32,
                               vx_image* const* out_i16, const vx_sgm_config* cfgs,
                               vx_stream stream);

/* No counterpart in the reference (its compute_disparity allocates per call,
 * vx-vision/src/kernels/sgm.rs:122-129). For callers that cannot allocate
 * device memory when they call - a host that owns all GPU memory through its
 * own allocator, a real-time loop that must not take the implicit device
 * synchronisation of cudaMalloc/cudaFree, a plugin whose host forbids
 * allocation during a call: same result as vx_sgm_compute_disparity, but all
 * intermediate state lives in a static device array of
 * vx_sgm_static_scratch_bytes() (64 MiB, held on every GPU where the library's
 * module is loaded until the process exits) and the call allocates nothing.
 * Planes are device pointers with pitches in bytes on the calling thread's
 * current device; out_i16 may be NULL. Pairs whose workspace does not fit are
 * rejected with VX_ERR_BUDGET. All calls share the array: calls whose GPU work
 * overlaps race on it. The first call on a device sets that device up; make it
 * before any stream capture. NULL stream = legacy default stream, synchronous. */
vx_status vx_sgm_compute_disparity_noalloc(const uint8_t* left, size_t left_pitch,
                                           const uint8_t* right, size_t right_pitch,
                                           uint32_t width, uint32_t height, float* out_f32,
                                           size_t out_f32_pitch, int16_t* out_i16,
                                           size_t out_i16_pitch, const vx_sgm_config* cfg,
                                           vx_stream stream);
/* Size in bytes of the static scratch used by vx_sgm_compute_disparity_noalloc. */
size_t vx_sgm_static_scratch_bytes(void);

/* Autotuner (no reference counterpart): runs this batch once per candidate
 * of the path-aggregation launch - both forms (32-scanline units on the
 * single-scanline kernel, 64-scanline units on the scanline-pair kernel) and
 * every warpgroups-per-CTA shape of each - `iterations` timed runs each (CUDA
 * events on the context's stream, one untimed run first), and records the
 * fastest for batches with the same key (largest padded D, census word width,
 * slab format, log2 of the queued 32-scanline units). Outputs are written like
 * vx_sgm_compute_batch. best_* may be NULL. Synchronous. */
vx_status vx_sgm_autotune_batch(vx_sgm* sgm, vx_ctx* ctx, uint32_t n, const vx_image* const* left,
                                const vx_image* const* right, vx_image* const* out_f32,
                                vx_image* const* out_i16, const vx_sgm_config* cfgs,
                                uint32_t iterations, uint32_t* best_warpgroups, float* best_ms,
                                uint32_t* best_unit_scanlines);
/* Persist / restore the autotuned table as JSON. */
vx_status vx_sgm_tuning_save(vx_sgm* sgm, const char* path);
vx_status vx_sgm_tuning_load(vx_sgm* sgm, const char* path);

/* CUDA graphs per shape bucket (no reference counterpart). With max_buckets
 * > 0, vx_sgm_compute_batch / compute_disparity keep, per bucket (the ordered
 * list of the pairs' sizes and configs), a resident workspace and a captured
 * graph of the launch sequence; a call of a known bucket refreshes the pair
 * table and launches the graph. At most max_buckets buckets are kept (least
 * recently used first out); 0 disables the cache and frees it. Calls of one
 * bucket share its workspace, so they must be ordered on one stream. */
vx_status vx_sgm_set_graph_cache(vx_sgm* sgm, uint32_t max_buckets);

/* Device bytes of intermediate state one pair needs (census, path slabs and the
 * matching-cost volume of the scanline-pair kernel). */
size_t vx_sgm_workspace_bytes(uint32_t width, uint32_t height, const vx_sgm_config* cfg);

/* Debug dump for parity tests (no reference counterpart): runs one pair and
 * copies to host the census words (u64 per pixel, may be NULL), the per-path
 * aggregated costs L_r (num_paths * H * W * D u16, HWD per path, may be
 * NULL) and the summed cost volume S (H * W * D u16, may be NULL). */
vx_status vx_sgm_debug_dump(vx_sgm* sgm, vx_ctx* ctx, const vx_image* left, const vx_image* right,
                            const vx_sgm_config* cfg, uint64_t* census_left,
                            uint64_t* census_right, uint16_t* path_costs, uint16_t* cost_volume);

/* Per-stage device timing (no reference counterpart; the reference only times
 * whole calls with Instant, examples/depth_to_cloud_demo.rs:48-53). Enabling
 * (re)starts a record: every later batch records CUDA events on its stream
 * around its census, cost-volume, path aggregation and WTA launches (the first
 * 256 batches are kept; batches run by the single-scanline kernel have no
 * cost-volume launch, its time is 0). vx_ctx_stage_times waits for those
 * events and returns the mean duration per batch of each stage in
 * milliseconds, census_ms covering the census and the cost volume
 * (VX_ERR_NOT_READY when no batch ran since timing was enabled);
 * vx_ctx_stage_times_detail returns the cost volume on its own. */
vx_status vx_ctx_enable_stage_timing(vx_ctx* ctx, int enable);
vx_status vx_ctx_stage_times(vx_ctx* ctx, float* census_ms, float* aggregate_ms, float* wta_ms);
vx_status vx_ctx_stage_times_detail(vx_ctx* ctx, float* census_ms, float* costs_ms, float* aggregate_ms,
                                    float* wta_ms);

/* ---- Serving loop (no reference counterpart) ----------------------------
 * Continuous batching of stereo requests of any size and config under a
 * device-memory budget. Creating the server takes a device arena of exactly
 * memory_budget_bytes from the context's pool and a pinned host staging arena
 * of host_staging_bytes (0: budget / 16, clamped to 256 MB .. 4 GB); serving
 * then allocates from these alone. submit() copies the images into the staging
 * arena and queues the request; a scheduler thread admits queued requests in
 * arrival order while an upper bound of their device bytes (workspace + images
 * + outputs + plan tables) fits the largest free block of the arena, batches up
 * to max_batch of them into one block, and runs the batch on one of
 * max_inflight_batches streams (upload, batched SGM, download); batches on
 * different streams overlap, and new requests join the next batch as soon as a
 * stream and memory are free. A request's result does not depend on the other
 * requests of its batch. A request larger than the whole budget is rejected
 * with VX_ERR_BUDGET. */
typedef struct vx_sgm_server vx_sgm_server;
typedef struct vx_server_config {
    size_t memory_budget_bytes;
    uint32_t max_batch;
    uint32_t max_inflight_batches;
    size_t host_staging_bytes;            /* 0 = default */
} vx_server_config;
typedef struct vx_server_stats {
    uint64_t submitted, completed, rejected, cancelled, failed, batches;
    uint64_t queued;                      /* waiting for admission */
    uint64_t inflight_bytes;              /* device arena bytes held by running batches */
    uint64_t completed_pixel_disparities; /* sum of W*H*D of completed requests */
    uint64_t pool_reserved_bytes;         /* device memory the context's pool holds */
    uint64_t pinned_bytes;                /* pinned host memory held (arena + overflow) */
    uint64_t max_launch_us;               /* longest host time to issue one batch */
    uint64_t max_pinned_alloc_us;         /* longest pinned allocation past the arena */
    uint64_t staging_overflows;           /* requests staged past the pinned arena */
    uint64_t shadow_reruns;               /* requests recomputed after their escape pool ran out */
    uint64_t max_batches_in_flight;       /* most batches unfinished on the GPU at once, counted
                                             when a batch is launched (itself included) */
} vx_server_stats;

vx_status vx_sgm_server_create(vx_sgm* sgm, vx_ctx* ctx, const vx_server_config* cfg,
                               vx_sgm_server** out);
/* Stops admitting, cancels queued requests, waits for running ones. */
void vx_sgm_server_destroy(vx_sgm_server* server);
/* left/right: host u8 planes (host_pitch bytes per row, 0 = width). */
vx_status vx_sgm_server_submit(vx_sgm_server* server, const uint8_t* left, const uint8_t* right,
                               uint32_t width, uint32_t height, size_t host_pitch,
                               const vx_sgm_config* cfg, int want_i16, uint64_t* request_id);
/* Waits up to timeout_ms (0 = poll: VX_ERR_NOT_READY if not done) and copies the
 * result (W*H f32, optional W*H i16) and the submit-to-completion latency out;
 * the request is then forgotten. VX_ERR_TIMEOUT when the wait runs out. */
vx_status vx_sgm_server_wait(vx_sgm_server* server, uint64_t request_id, float* disparity,
                             int16_t* disparity_i16, double* latency_ms, uint32_t timeout_ms);
/* Cancels a request that is still queued (VX_ERR_NOT_READY once it started). */
vx_status vx_sgm_server_cancel(vx_sgm_server* server, uint64_t request_id);
vx_status vx_sgm_server_get_stats(vx_sgm_server* server, vx_server_stats* out);

/* ---- Depth-map post-filters (vx-vision/src/kernels/depth_filter.rs) -------
 * The step after WTA in vx-vision's depth chain. Both read an F32 image and
 * write another F32 image of the same size (they must differ); NULL stream =
 * the context's stream, synchronous (the reference's apply_* wait for their
 * command buffer); otherwise asynchronous on that stream (encode_*). */
/* DepthFilterConfig (depth_filter.rs:19-49): defaults radius 3, sigma_spatial
 * 5.0, sigma_depth 0.05. Validated: radius 0..32, sigmas finite and > 0. */
typedef struct vx_depth_filter_config {
    int32_t radius;
    float sigma_spatial;
    float sigma_depth;
} vx_depth_filter_config;
/* DepthMedianConfig (depth_filter.rs:51-63): default radius 1 (3x3).
 * Validated: radius 0..5 (the shader's window array holds 121 values). */
typedef struct vx_depth_median_config {
    int32_t radius;
} vx_depth_median_config;
void vx_depth_filter_config_default(vx_depth_filter_config* cfg);
void vx_depth_median_config_default(vx_depth_median_config* cfg);
typedef struct vx_depth_filter vx_depth_filter;
/* Replaces DepthFilter::new(&ctx) (depth_filter.rs:76-100). */
vx_status vx_depth_filter_create(vx_ctx* ctx, vx_depth_filter** out);
void vx_depth_filter_destroy(vx_depth_filter* filter);
/* Replaces DepthFilter::apply_median / encode_median (depth_filter.rs:140-232):
 * per pixel, the median (upper middle for an even count) of the window's
 * values > 0, clamped coordinates; 0 where none is valid
 * (DepthFilter.metal:84-120). Invalid SGM pixels (value <= 0) are left out. */
vx_status vx_depth_filter_apply_median(vx_depth_filter* filter, vx_ctx* ctx, const vx_image* in,
                                       vx_image* out, const vx_depth_median_config* cfg,
                                       vx_stream stream);
/* Replaces DepthFilter::apply_bilateral / encode_bilateral (depth_filter.rs:
 * 102-203): edge-preserving weighted mean of the valid neighbours
 * (DepthFilter.metal:20-66); 0 where the centre is <= 0. */
vx_status vx_depth_filter_apply_bilateral(vx_depth_filter* filter, vx_ctx* ctx, const vx_image* in,
                                          vx_image* out, const vx_depth_filter_config* cfg,
                                          vx_stream stream);

/* ---- Sparse ORB stereo matching (vx-vision/src/kernels/stereomatch.rs) -----
 * For each left keypoint, the right keypoint with the smallest Hamming distance
 * between their 256-bit ORB descriptors among those passing the epipolar test
 * |yl - yr| <= max_epipolar and min_disparity <= xl - xr <= max_disparity; the
 * first in right index order on ties (StereoMatch.metal:32-93). Accepted when
 * the distance is <= max_hamming cast to 16 bits (StereoMatch.metal:96; the
 * Lowe ratio test there is commented out, so ratio_thresh is carried but
 * unused), then triangulated: Z = fx*baseline/d, X = Z*(xl-cx)/fx,
 * Y = Z*(yl-cy)/fy in IEEE single precision, that operation order. A left
 * keypoint with no candidate is matched to right index 0 only when max_hamming
 * is 0xFFFF (the shader's initial best). Matches come out in ascending left
 * index (the reference's atomic append leaves their order unspecified).
 * Calls on one matcher must be ordered (one stream, or synchronised between):
 * they share its scratch. */
/* CornerPoint (vx-vision/src/types.rs:8-12): 16 bytes. */
typedef struct vx_corner_point {
    float position[2];
    float response;
    uint32_t pyramid_level;
} vx_corner_point;
/* ORBOutput (types.rs:36-39): 256-bit descriptor and angle, 36 bytes. */
typedef struct vx_orb_output {
    uint32_t desc[8];
    float angle;
} vx_orb_output;
/* StereoMatchResult as the reference's host reads it (types.rs:64-70), 28 bytes;
 * _pad is 0. */
typedef struct vx_stereo_match_result {
    uint32_t left_idx;
    uint32_t right_idx;
    float disparity;
    float point_3d[3];
    float _pad;
} vx_stereo_match_result;
/* StereoConfig (stereomatch.rs:19-69). Defaults: max_epipolar 2, min_disparity
 * 1, max_disparity 120, max_hamming 50, ratio_thresh 0.8, fx = fy = 600,
 * cx 320, cy 240, baseline 0.12. Every value is accepted, as the reference does. */
typedef struct vx_stereo_config {
    float max_epipolar;
    float min_disparity;
    float max_disparity;
    uint32_t max_hamming;
    float ratio_thresh;
    float fx, fy, cx, cy;
    float baseline;
} vx_stereo_config;
void vx_stereo_config_default(vx_stereo_config* cfg);
typedef struct vx_stereo_matcher vx_stereo_matcher;
/* Replaces StereoMatcher::new(&ctx) (stereomatch.rs:84-112). */
vx_status vx_stereo_matcher_create(vx_ctx* ctx, vx_stereo_matcher** out);
void vx_stereo_matcher_destroy(vx_stereo_matcher* matcher);
/* Replaces StereoMatcher::run (stereomatch.rs:115-249): host arrays in, host
 * array out, synchronous. Keypoint and descriptor counts must agree per side
 * (the reference asserts), capacity >= n_left_kpts; at most 2^26 left and
 * 2^23 - 1 right keypoints. *n_matches receives the number of records. */
vx_status vx_stereo_matcher_run(vx_stereo_matcher* matcher, vx_ctx* ctx, const vx_corner_point* left_kpts,
                                size_t n_left_kpts, const vx_corner_point* right_kpts, size_t n_right_kpts,
                                const vx_orb_output* left_descs, size_t n_left_descs,
                                const vx_orb_output* right_descs, size_t n_right_descs,
                                const vx_stereo_config* cfg, vx_stereo_match_result* matches, size_t capacity,
                                size_t* n_matches);
/* The same on device memory, for pipelines whose keypoints and descriptors
 * are already on the GPU (the buffers run() uploads, stereomatch.rs:144-169):
 * descriptors as 8 words per keypoint; keypoints and descriptors 16-byte
 * aligned; matches has room for n_left records; *match_count (device) gets
 * their number. NULL stream = the context's stream, synchronous. */
vx_status vx_stereo_matcher_run_device(vx_stereo_matcher* matcher, vx_ctx* ctx, const vx_corner_point* left_kpts,
                                       uint32_t n_left, const vx_corner_point* right_kpts, uint32_t n_right,
                                       const uint32_t* left_desc_words, const uint32_t* right_desc_words,
                                       const vx_stereo_config* cfg, vx_stereo_match_result* matches,
                                       uint32_t* match_count, vx_stream stream);

/* Many frames in one launch (an addition for callers that match every frame of
 * a sequence; per frame the result of run()): the keypoints and descriptors of
 * all frames concatenated on the device, frame f's left keypoints at
 * [left_offsets[f], left_offsets[f+1]) and right ones likewise (host arrays of
 * n_frames + 1, starting at 0, non-decreasing; at most 2^23 - 1 right keypoints
 * a frame). Frame f's matches go to matches + left_offsets[f] in ascending left
 * index with frame-relative indices; match_counts[f] (device) gets their
 * number. One CTA per frame: for frames of up to a few thousand keypoints.
 * NULL stream = the context's stream, synchronous. */
vx_status vx_stereo_matcher_run_frames_device(vx_stereo_matcher* matcher, vx_ctx* ctx, uint32_t n_frames,
                                              const uint32_t* left_offsets, const uint32_t* right_offsets,
                                              const vx_corner_point* left_kpts, const vx_corner_point* right_kpts,
                                              const uint32_t* left_desc_words, const uint32_t* right_desc_words,
                                              const vx_stereo_config* cfg, vx_stereo_match_result* matches,
                                              uint32_t* match_counts, vx_stream stream);

/* ---- The depth chain around SGM: colour ingest and point clouds ----------
 * Replaces ColorConvert::rgba_to_gray (vx-vision/src/kernels/color.rs:62,
 * ColorConvert.metal:21-32): in RGBA8, out U8 of the same size; gray =
 * 0.299 r + 0.587 g + 0.114 b on the unorm values (byte / 255) in single
 * precision, in that order, stored as an 8-bit unorm (clamp to [0, 1], x 255,
 * round to nearest even). The gray image feeds vx_sgm_compute_disparity.
 * NULL stream = the context's stream, synchronous. */
vx_status vx_color_rgba_to_gray(vx_ctx* ctx, const vx_image* in, vx_image* out, vx_stream stream);

/* DepthToCloudConfig (vx-vision/src/kernels/depth_to_cloud.rs:23-59). Defaults:
 * min_depth 0.1, max_depth 10, depth_scale 1, max_points 1 000 000. */
typedef struct vx_depth_to_cloud_config {
    float min_depth;
    float max_depth;
    float depth_scale;
    uint32_t max_points;
} vx_depth_to_cloud_config;
void vx_depth_to_cloud_config_default(vx_depth_to_cloud_config* cfg);
/* GpuPoint3D (vx-vision/src/types.rs:440-448), 36 bytes: the records the
 * reference's PointCloud::from_gpu_points reads (types_3d.rs:63-73). */
typedef struct vx_point3d {
    float position[3];
    float _pad0;
    uint8_t color[4];
    float normal[3];
    float _pad1;
} vx_point3d;
typedef struct vx_depth_to_cloud vx_depth_to_cloud;
/* Replaces DepthToCloud::new(&ctx) (depth_to_cloud.rs:66-80). */
vx_status vx_depth_to_cloud_create(vx_ctx* ctx, vx_depth_to_cloud** out);
void vx_depth_to_cloud_destroy(vx_depth_to_cloud* dc);
/* Replaces DepthToCloud::compute_raw (depth_to_cloud.rs:104-188,
 * DepthToCloud.metal:30-70): every pixel of the F32 depth map with d = depth *
 * depth_scale inside [min_depth, max_depth] (NaN passes, as in the shader)
 * becomes the point ((x - cx) d / fx, (y - cy) d / fy, d) (IEEE single
 * precision, that order), colour (r, g, b, 255) from an RGBA8 color image,
 * (v, 0, 0, 255) from a U8 one, (255, 255, 255, 255) when color is NULL or at
 * most 1 pixel wide (the shader's test), normal 0. color must otherwise be the
 * depth map's size. At most min(max_points, W*H) points, in row-major pixel
 * order (the reference appends them atomically, in no fixed order); points
 * must hold that many; *n_points gets their number. Synchronous. */
vx_status vx_depth_to_cloud_compute_raw(vx_depth_to_cloud* dc, vx_ctx* ctx, const vx_image* depth,
                                        const vx_image* color, float fx, float fy, float cx, float cy,
                                        const vx_depth_to_cloud_config* cfg, vx_point3d* points, size_t capacity,
                                        size_t* n_points);
/* Replaces DepthToCloud::compute (depth_to_cloud.rs:86-101): compute_raw with
 * the depth map's intrinsics (for example the DepthMap of vx_sgm_compute with
 * its depth output). */
vx_status vx_depth_to_cloud_compute(vx_depth_to_cloud* dc, vx_ctx* ctx, const vx_depth_map* depth,
                                    const vx_image* color, const vx_depth_to_cloud_config* cfg, vx_point3d* points,
                                    size_t capacity, size_t* n_points);
/* The same on device memory (an addition for pipelines that keep the cloud on
 * the GPU): the first min(max_points, W*H, capacity) points go to d_points,
 * and *d_count (device) gets the number of pixels that passed (which may exceed
 * it, like the reference's count buffer). Buffers 4-byte aligned. NULL stream =
 * the context's stream, synchronous; otherwise asynchronous. Calls on one
 * handle must be ordered (they share its tile counts). */
vx_status vx_depth_to_cloud_compute_device(vx_depth_to_cloud* dc, vx_ctx* ctx, const vx_image* depth,
                                           const vx_image* color, float fx, float fy, float cx, float cy,
                                           const vx_depth_to_cloud_config* cfg, vx_point3d* d_points,
                                           uint32_t capacity, uint32_t* d_count, vx_stream stream);

/* Number of this library's kernel launches issued since load (all threads). */
uint64_t vx_kernel_launch_count(void);
/* Number of memory allocations this library has requested since load (all
 * threads): device pool allocations, cudaMalloc*, pinned host cudaMallocHost.
 * Lets a caller check that a call allocated nothing. */
uint64_t vx_memory_allocation_count(void);

#ifdef __cplusplus
}
#endif
#endif /* VX_SGM_H */
