// Sparse ORB stereo matching (vx-vision's StereoMatcher: kernels/stereomatch.rs,
// shaders/StereoMatch.metal). For every left keypoint: the right keypoint of
// smallest Hamming distance between 256-bit descriptors among those on the same
// epipolar line (|yl - yr| <= max_epipolar) within the disparity range
// (min_disparity <= xl - xr <= max_disparity), the first one in right index
// order on ties; accepted when that distance is at most max_hamming (cast to
// 16 bits, as the shader's ushort(params.max_hamming)); then triangulated.
// A left keypoint without any candidate takes right index 0 at distance 0xFFFF
// (StereoMatch.metal:79-96), which only a max_hamming of 0xFFFF accepts.
//
// The reference writes the n_left x n_right u16 distance matrix to memory and
// scans each row in a second kernel. Here a row is reduced while it is produced:
//   match_kernel  grid (left tiles of 256, right chunks). One thread per left
//                 keypoint (descriptor in registers); the CTA stages its chunk of
//                 right positions and descriptors in shared memory and every
//                 thread scans it: the epipolar and disparity tests in float, the
//                 distance (8 x LOP3 + POPC) only where both pass, and a running
//                 minimum of key = distance << 23 | right index, whose minimum is
//                 the first minimum in right index order. With several chunks per
//                 tile the keys meet in global memory by atomicMin; the CTA that
//                 arrives last at its tile (fence + arrival counter, no waiting)
//                 decides the tile's matches and stores their count.
//   emit_kernel   one CTA per 1024 left keypoints: the tile counts before it give
//                 its output offset, a block scan of its accept flags the slots;
//                 triangulation in the shader's operation order with IEEE
//                 round-to-nearest (no fused multiply-add), then the record. It
//                 resets the keys for the next call, the last CTA stores the count.
// The matches come out in ascending left index (the reference appends through
// an atomic counter, so its order is unspecified; the records are the same).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "launch.hpp"

namespace vxsgm {

namespace {

constexpr int kTileLefts = 256;     // left keypoints (threads) per match CTA
constexpr int kStage = 512;         // right keypoints staged in shared memory per pass
constexpr int kEmitThreads = 1024;  // left keypoints per emit CTA
constexpr int kRightBits = 23;
constexpr uint32_t kRightMask = (1u << kRightBits) - 1u;
constexpr uint32_t kNoKey = 0xFFFFFFFFu;

__device__ __forceinline__ uint32_t hamming256(const uint4& a0, const uint4& a1, const uint4& b0,
                                               const uint4& b1) {
    return __popc(a0.x ^ b0.x) + __popc(a0.y ^ b0.y) + __popc(a0.z ^ b0.z) + __popc(a0.w ^ b0.w) +
           __popc(a1.x ^ b1.x) + __popc(a1.y ^ b1.y) + __popc(a1.z ^ b1.z) + __popc(a1.w ^ b1.w);
}

// Whether the match of a final key passes the distance threshold; a key that
// saw no candidate stands for the shader's initial best = 0xFFFF
// (StereoMatch.metal:79-96).
__device__ __forceinline__ bool accepted(uint32_t key, uint32_t max_ham) {
    const uint32_t dist = key == kNoKey ? 0xFFFFu : key >> kRightBits;
    return dist <= max_ham;
}

__global__ void __launch_bounds__(kTileLefts) match_kernel(const float4* __restrict__ lk,
                                                           const float4* __restrict__ rk,
                                                           const uint4* __restrict__ ld,
                                                           const uint4* __restrict__ rd, uint32_t* keys,
                                                           uint32_t* arrivals, uint32_t* tile_counts,
                                                           StereoMatchParams p) {
    __shared__ float2 s_pos[kStage];
    __shared__ uint4 s_desc[2 * kStage];
    __shared__ int s_last;

    const uint32_t tile = blockIdx.x;
    const uint32_t li = tile * kTileLefts + threadIdx.x;
    const bool have = li < p.n_left;
    // A thread past the last left keypoint scans with y = NaN: no test passes.
    float lx = 0.0f, ly = __int_as_float(0x7fc00000);
    uint4 a0 = make_uint4(0, 0, 0, 0), a1 = a0;
    if (have) {
        const float4 k = lk[li];
        lx = k.x;
        ly = k.y;
        a0 = ld[2 * (size_t)li];
        a1 = ld[2 * (size_t)li + 1];
    }

    uint32_t best = kNoKey;
    const uint32_t r_begin = blockIdx.y * p.chunk;
    const uint32_t r_end = min(p.n_right, r_begin + p.chunk);
    for (uint32_t base = r_begin; base < r_end; base += kStage) {
        const uint32_t cnt = min((uint32_t)kStage, r_end - base);
        __syncthreads();  // the previous stage has been read
        for (uint32_t k = threadIdx.x; k < cnt; k += kTileLefts) {
            const float4 q = rk[base + k];
            s_pos[k] = make_float2(q.x, q.y);
        }
        for (uint32_t k = threadIdx.x; k < 2 * cnt; k += kTileLefts) s_desc[k] = rd[2 * (size_t)base + k];
        __syncthreads();
#pragma unroll 4
        for (uint32_t k = 0; k < cnt; ++k) {
            const float2 q = s_pos[k];
            const float dy = fabsf(__fsub_rn(ly, q.y));
            const float d = __fsub_rn(lx, q.x);
            if (dy <= p.max_epipolar && d >= p.min_disparity && d <= p.max_disparity) {
                const uint32_t dist = hamming256(a0, a1, s_desc[2 * k], s_desc[2 * k + 1]);
                best = min(best, (dist << kRightBits) | (base + k));
            }
        }
    }

    uint32_t key = best;
    if (p.splits > 1) {
        if (have && best != kNoKey) atomicMin(&keys[li], best);
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0) s_last = atomicAdd(&arrivals[tile], 1u) == p.splits - 1;
        __syncthreads();
        if (!s_last) return;
        __threadfence();
        if (have) key = __ldcg(&keys[li]);
    } else if (have) {
        keys[li] = key;
    }
    const int n = __syncthreads_count(have && accepted(key, p.max_hamming));
    if (threadIdx.x == 0) {
        tile_counts[tile] = (uint32_t)n;
        if (p.splits > 1) arrivals[tile] = 0;  // ready for the next call
    }
}

__global__ void __launch_bounds__(kEmitThreads) emit_kernel(const float4* __restrict__ lk,
                                                            const float4* __restrict__ rk, uint32_t* keys,
                                                            const uint32_t* __restrict__ tile_counts,
                                                            StereoMatchRecord* __restrict__ out,
                                                            uint32_t* __restrict__ count, StereoMatchParams p,
                                                            uint32_t tiles_per_cta) {
    __shared__ uint32_t s_warp[kEmitThreads / 32];
    __shared__ uint32_t s_prefix;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

    // Matches of the tiles before this CTA's first tile.
    const uint32_t first_tile = blockIdx.x * tiles_per_cta;
    uint32_t acc = 0;
    for (uint32_t t = threadIdx.x; t < first_tile; t += kEmitThreads) acc += tile_counts[t];
    acc = __reduce_add_sync(0xffffffffu, acc);
    if (lane == 0) s_warp[warp] = acc;
    __syncthreads();
    if (warp == 0) {
        uint32_t v = s_warp[lane];
        v = __reduce_add_sync(0xffffffffu, v);
        if (lane == 0) s_prefix = v;
    }
    __syncthreads();
    const uint32_t prefix = s_prefix;

    const uint32_t li = blockIdx.x * kEmitThreads + threadIdx.x;
    uint32_t key = kNoKey;
    if (li < p.n_left) {
        key = keys[li];
        keys[li] = kNoKey;  // ready for the next call
    }
    const bool take = li < p.n_left && accepted(key, p.max_hamming);
    const uint32_t ballot = __ballot_sync(0xffffffffu, take);
    __syncthreads();  // s_warp reused
    if (lane == 0) s_warp[warp] = __popc(ballot);
    __syncthreads();
    if (warp == 0) {
        const uint32_t v = s_warp[lane];
        uint32_t incl = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        s_warp[lane] = incl - v;
        if (blockIdx.x == gridDim.x - 1 && lane == 31) *count = prefix + incl;
    }
    __syncthreads();
    if (!take) return;
    const uint32_t slot = prefix + s_warp[warp] + __popc(ballot & ((1u << lane) - 1u));
    const uint32_t ri = key == kNoKey ? 0u : (key & kRightMask);
    const float4 l = lk[li];
    const float4 r = rk[ri];
    // StereoMatch.metal:104-107, operation for operation.
    const float disp = __fsub_rn(l.x, r.x);
    const float Z = __fdiv_rn(__fmul_rn(p.fx, p.baseline), disp);
    const float X = __fdiv_rn(__fmul_rn(Z, __fsub_rn(l.x, p.cx)), p.fx);
    const float Y = __fdiv_rn(__fmul_rn(Z, __fsub_rn(l.y, p.cy)), p.fy);
    StereoMatchRecord& o = out[slot];
    o.left_idx = li;
    o.right_idx = ri;
    o.disparity = disp;
    o.point_3d[0] = X;
    o.point_3d[1] = Y;
    o.point_3d[2] = Z;
    o.pad = 0.0f;
}

// ---- banded form: right keypoints bucketed by image row --------------------
//
// Only right keypoints within max_epipolar rows of a left keypoint can pass the
// epipolar test, so for large sets the right keypoints are counting-sorted into
// 1-pixel row buckets (rows 0..kRowBuckets-1; everything else, NaN and
// infinities included, into one extra "special" bucket) and each left keypoint
// scans the rows floor(fl(y - e)) - 1 .. floor(fl(y + e)) + 1 (less the outer
// two where the test provably fails there) plus the special bucket. That range holds every right keypoint the exact test can accept when
// |y| < 2^22 and 0 <= e < 2^20: then |y - yr| and y +- e stay below 2^23, where
// single-precision rounding moves a difference by at most 0.25, so
// fl(|y - yr|) <= e implies yr in [fl(y - e) - 0.5, fl(y + e) + 0.5]. A left
// keypoint with |y| >= 2^22 (or NaN, infinite) scans the special bucket only,
// which holds every right keypoint it could pass with. The host uses this form
// only for e in [0, 2^20). Keys carry the original right index, so the minimum
// does not depend on the bucket order (which the scatter's atomics leave open).

constexpr int kBandThreads = 256;               // threads per banded CTA
constexpr int kBandLefts = kBandThreads / 32;    // left keypoints (one warp each) per banded CTA
static_assert(kTileLefts % kBandLefts == 0, "a banded CTA's keypoints lie in one tile");
constexpr int kCountThreads = 256;

__device__ __forceinline__ uint32_t row_bucket(float y) {
    return (y >= 0.0f && y < (float)kRowBuckets) ? (uint32_t)y : (uint32_t)kRowBuckets;
}

// Counts the right keypoints per row bucket in `hist` (device atomics) and
// zeroes the tile counts the banded match accumulates into. The last CTA to
// arrive (the pattern of a cooperative grid barrier: CTA barrier, then one
// thread fences and takes a ticket; nothing waits) turns the counts into
// bucket starts (row_start[0..kRowBuckets+1], the last = n_right) and scatter
// cursors, and leaves hist and the arrival counter at 0. Its scan stages the
// counts in shared memory so that global reads and writes stay coalesced; each
// thread sums a run of kPer (odd) consecutive words, which no two lanes of a
// warp read from the same bank.
__global__ void __launch_bounds__(kCountThreads) bucket_count_kernel(const float4* __restrict__ rk,
                                                                     uint32_t n_right, uint32_t* hist,
                                                                     uint32_t* arrival, uint32_t* row_start,
                                                                     uint32_t* cursor, uint32_t* tile_counts,
                                                                     uint32_t n_tiles) {
    constexpr int kPer = (kRowBuckets + 1 + kCountThreads - 1) / kCountThreads;
    static_assert(kPer % 2 == 1, "odd run length keeps the runs on distinct banks");
    static_assert(kPer * kCountThreads > kRowBuckets + 1, "room for the total past the counts");
    __shared__ uint32_t s_cnt[kPer * kCountThreads];
    __shared__ uint32_t s_warp[kCountThreads / 32];
    __shared__ int s_last;
    const uint32_t k = blockIdx.x * kCountThreads + threadIdx.x;
    if (k < n_right) atomicAdd(&hist[row_bucket(rk[k].y)], 1u);
    for (uint32_t t = k; t < n_tiles; t += gridDim.x * kCountThreads) tile_counts[t] = 0;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = atomicAdd(arrival, 1u) == gridDim.x - 1;
        if (s_last) __threadfence();
    }
    __syncthreads();
    if (!s_last) return;

    {
        uint32_t v[kPer];  // all loads in flight before the first store
#pragma unroll
        for (int i = 0; i < kPer; ++i) {
            const int b = threadIdx.x + i * kCountThreads;
            v[i] = b <= kRowBuckets ? __ldcg(&hist[b]) : 0u;
        }
#pragma unroll
        for (int i = 0; i < kPer; ++i) s_cnt[threadIdx.x + i * kCountThreads] = v[i];
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t* run_at = s_cnt + threadIdx.x * kPer;
    uint32_t run = 0;
#pragma unroll
    for (int i = 0; i < kPer; ++i) run += run_at[i];
    uint32_t incl = run;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        const uint32_t w = lane < kCountThreads / 32 ? s_warp[lane] : 0u;
        uint32_t wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += t;
        }
        if (lane < kCountThreads / 32) s_warp[lane] = wi - w;
    }
    __syncthreads();
    uint32_t start = s_warp[warp] + incl - run;
#pragma unroll
    for (int i = 0; i < kPer; ++i) {
        const uint32_t c = run_at[i];
        run_at[i] = start;
        start += c;
    }
    __syncthreads();
    // Entry kRowBuckets + 1 (a zero past the counts) now holds the total.
    for (int b = threadIdx.x; b <= kRowBuckets + 1; b += kCountThreads) {
        row_start[b] = s_cnt[b];
        if (b <= kRowBuckets) {
            cursor[b] = s_cnt[b];
            hist[b] = 0;  // ready for the next call
        }
    }
    if (threadIdx.x == 0) *arrival = 0;
}

__global__ void __launch_bounds__(256) bucket_scatter_kernel(const float4* __restrict__ rk,
                                                             const uint4* __restrict__ rd, uint32_t n_right,
                                                             uint32_t* cursor, float2* __restrict__ s_pos,
                                                             uint4* __restrict__ s_desc, uint32_t* __restrict__ s_idx) {
    const uint32_t k = blockIdx.x * 256 + threadIdx.x;
    if (k >= n_right) return;
    const float4 q = rk[k];
    const uint32_t at = atomicAdd(&cursor[row_bucket(q.y)], 1u);
    s_pos[at] = make_float2(q.x, q.y);
    s_desc[2 * (size_t)at] = rd[2 * (size_t)k];
    s_desc[2 * (size_t)at + 1] = rd[2 * (size_t)k + 1];
    s_idx[at] = k;
}

// The lanes of a warp take every 32nd right keypoint of [r0, r1).
__device__ __forceinline__ uint32_t scan_range(uint32_t best, uint32_t r0, uint32_t r1, uint32_t lane, float lx,
                                               float ly, const uint4& a0, const uint4& a1,
                                               const float2* __restrict__ s_pos, const uint4* __restrict__ s_desc,
                                               const uint32_t* __restrict__ s_idx, float max_epipolar,
                                               float min_disparity, float max_disparity) {
    for (uint32_t k = r0 + lane; k < r1; k += 32) {
        const float2 q = s_pos[k];
        const float dy = fabsf(__fsub_rn(ly, q.y));
        const float d = __fsub_rn(lx, q.x);
        if (dy <= max_epipolar && d >= min_disparity && d <= max_disparity) {
            const uint4* b = s_desc + 2 * k;
            const uint32_t dist = hamming256(a0, a1, b[0], b[1]);
            best = min(best, (dist << kRightBits) | s_idx[k]);
        }
    }
    return best;
}

// One warp per left keypoint, kBandLefts keypoints per CTA: the warp scans the
// keypoint's band of rows, then the special bucket, with coalesced reads of the
// sorted copies, and takes the minimum over its lanes. The CTA adds its
// matches to the count of its 256-keypoint tile (zeroed by the count kernel).
__global__ void __launch_bounds__(kBandThreads) match_banded_kernel(
    const float4* __restrict__ lk, const uint4* __restrict__ ld, const uint32_t* __restrict__ row_start,
    const float2* __restrict__ s_pos, const uint4* __restrict__ s_desc, const uint32_t* __restrict__ s_idx,
    uint32_t* keys, uint32_t* tile_counts, StereoMatchParams p) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t li = blockIdx.x * kBandLefts + (threadIdx.x >> 5);
    const bool have = li < p.n_left;
    uint32_t best = kNoKey;
    if (have) {
        const float4 l = lk[li];
        const uint4 a0 = ld[2 * (size_t)li], a1 = ld[2 * (size_t)li + 1];
        const float e = p.max_epipolar;  // the host guarantees 0 <= e < 2^20
        if (fabsf(l.y) < 4194304.0f) {   // 2^22
            // Rows floor(fl(y - e)) - 1 .. floor(fl(y + e)) + 1 hold every right
            // keypoint that can pass; the outer two are dropped when the test
            // already fails at their inner edge (the largest float below
            // floor(fl(y - e)), resp. floor(fl(y + e)) + 1): fl(|y - yr|) only
            // grows as yr moves outward, so no keypoint of that row can pass.
            const float fa = floorf(__fsub_rn(l.y, e)), fb = floorf(__fadd_rn(l.y, e));
            int lo = (int)fa - 1, hi = (int)fb + 1;
            if (fa >= 1.0f && !(fabsf(__fsub_rn(l.y, __int_as_float(__float_as_int(fa) - 1))) <= e)) ++lo;
            if (!(fabsf(__fsub_rn(l.y, fb + 1.0f)) <= e)) --hi;
            lo = max(lo, 0);
            hi = min(hi, kRowBuckets - 1);
            if (lo <= hi)
                best = scan_range(best, row_start[lo], row_start[hi + 1], lane, l.x, l.y, a0, a1, s_pos, s_desc,
                                  s_idx, e, p.min_disparity, p.max_disparity);
        }
        best = scan_range(best, row_start[kRowBuckets], row_start[kRowBuckets + 1], lane, l.x, l.y, a0, a1, s_pos,
                          s_desc, s_idx, e, p.min_disparity, p.max_disparity);
        best = __reduce_min_sync(0xffffffffu, best);  // `have` is uniform across the warp
    }
    const bool lead = have && lane == 0;
    if (lead) keys[li] = best;
    const int n = __syncthreads_count(lead && accepted(best, p.max_hamming));
    if (threadIdx.x == 0 && n) atomicAdd(&tile_counts[(blockIdx.x * kBandLefts) / kTileLefts], (uint32_t)n);
}

// ---- frames: many small keypoint sets in one launch -------------------------
//
// One CTA per frame (frame f: left keypoints [lo[f], lo[f+1]), right keypoints
// [ro[f], ro[f+1]) of the concatenated arrays). The CTA takes its left
// keypoints 256 at a time; for each such tile it stages the frame's right
// keypoints in shared memory as the match kernel does, keeps the running
// minimum key per thread, then emits the tile's matches in left index order
// (block scan) after those of the frame's earlier tiles. Records go to
// out[lo[f] + slot] with frame-relative indices; counts[f] gets the frame's
// number of matches. No scratch, no second kernel: for frames of up to a few
// thousand keypoints, where a launch per frame would cost more than its work.
__global__ void __launch_bounds__(kTileLefts) match_frames_kernel(
    const float4* __restrict__ lk, const float4* __restrict__ rk, const uint4* __restrict__ ld,
    const uint4* __restrict__ rd, const uint32_t* __restrict__ lo, const uint32_t* __restrict__ ro,
    StereoMatchRecord* __restrict__ out, uint32_t* __restrict__ counts, StereoMatchParams p) {
    __shared__ float2 s_pos[kStage];
    __shared__ uint4 s_desc[2 * kStage];
    __shared__ uint32_t s_warp[kTileLefts / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t f = blockIdx.x;
    const uint32_t l_begin = lo[f], nl = lo[f + 1] - l_begin;
    const uint32_t r_begin = ro[f], nr = ro[f + 1] - r_begin;
    uint32_t emitted = 0;
    for (uint32_t t0 = 0; t0 < nl; t0 += kTileLefts) {
        const uint32_t li = t0 + threadIdx.x;  // frame-relative
        const bool have = li < nl && nr > 0;
        float lx = 0.0f, ly = __int_as_float(0x7fc00000);
        uint4 a0 = make_uint4(0, 0, 0, 0), a1 = a0;
        if (have) {
            const float4 k = lk[l_begin + li];
            lx = k.x;
            ly = k.y;
            a0 = ld[2 * (size_t)(l_begin + li)];
            a1 = ld[2 * (size_t)(l_begin + li) + 1];
        }
        uint32_t best = kNoKey;
        for (uint32_t base = 0; base < nr; base += kStage) {
            const uint32_t cnt = min((uint32_t)kStage, nr - base);
            __syncthreads();
            for (uint32_t k = threadIdx.x; k < cnt; k += kTileLefts) {
                const float4 q = rk[r_begin + base + k];
                s_pos[k] = make_float2(q.x, q.y);
            }
            for (uint32_t k = threadIdx.x; k < 2 * cnt; k += kTileLefts)
                s_desc[k] = rd[2 * (size_t)(r_begin + base) + k];
            __syncthreads();
#pragma unroll 4
            for (uint32_t k = 0; k < cnt; ++k) {
                const float2 q = s_pos[k];
                const float dy = fabsf(__fsub_rn(ly, q.y));
                const float d = __fsub_rn(lx, q.x);
                if (dy <= p.max_epipolar && d >= p.min_disparity && d <= p.max_disparity) {
                    const uint32_t dist = hamming256(a0, a1, s_desc[2 * k], s_desc[2 * k + 1]);
                    best = min(best, (dist << kRightBits) | (base + k));
                }
            }
        }
        // A frame without right keypoints has no matches (stereomatch.rs:138-142).
        const bool take = have && accepted(best, p.max_hamming);
        const uint32_t ballot = __ballot_sync(0xffffffffu, take);
        __syncthreads();  // s_warp reused across tiles
        if (lane == 0) s_warp[warp] = __popc(ballot);
        __syncthreads();
        uint32_t before = 0, total = 0;
        for (int w = 0; w < kTileLefts / 32; ++w) {
            const uint32_t c = s_warp[w];
            before += w < warp ? c : 0u;
            total += c;
        }
        if (take) {
            const uint32_t slot = emitted + before + __popc(ballot & ((1u << lane) - 1u));
            const uint32_t ri = best == kNoKey ? 0u : (best & kRightMask);
            const float4 l = lk[l_begin + li];
            const float4 r = rk[r_begin + ri];
            const float disp = __fsub_rn(l.x, r.x);
            const float Z = __fdiv_rn(__fmul_rn(p.fx, p.baseline), disp);
            const float X = __fdiv_rn(__fmul_rn(Z, __fsub_rn(l.x, p.cx)), p.fx);
            const float Y = __fdiv_rn(__fmul_rn(Z, __fsub_rn(l.y, p.cy)), p.fy);
            StereoMatchRecord& o = out[l_begin + slot];
            o.left_idx = li;
            o.right_idx = ri;
            o.disparity = disp;
            o.point_3d[0] = X;
            o.point_3d[1] = Y;
            o.point_3d[2] = Z;
            o.pad = 0.0f;
        }
        emitted += total;
    }
    if (threadIdx.x == 0) counts[f] = emitted;
}

}  // namespace

cudaError_t launch_stereo_match_frames(const float4* left_kpts, const float4* right_kpts, const uint4* left_desc,
                                       const uint4* right_desc, const uint32_t* left_offsets,
                                       const uint32_t* right_offsets, uint32_t n_frames, StereoMatchRecord* out,
                                       uint32_t* counts, StereoMatchParams p, cudaStream_t stream) {
    if (n_frames == 0) return cudaSuccess;
    match_frames_kernel<<<n_frames, kTileLefts, 0, stream>>>(left_kpts, right_kpts, left_desc, right_desc,
                                                             left_offsets, right_offsets, out, counts, p);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) count_launch();
    return e;
}

StereoMatchShape stereo_match_shape(uint32_t n_left, uint32_t n_right, int sm_count) {
    StereoMatchShape s;
    s.left_tiles = (n_left + kTileLefts - 1) / kTileLefts;
    s.emit_ctas = (n_left + kEmitThreads - 1) / kEmitThreads;
    // About one wave of 256-thread CTAs (8 per SM), chunks of at least 256 rights.
    const uint64_t want = (uint64_t)sm_count * 8;
    uint64_t splits = (want + s.left_tiles - 1) / (s.left_tiles ? s.left_tiles : 1);
    const uint64_t max_splits = n_right / 256 > 0 ? n_right / 256 : 1;
    if (splits > max_splits) splits = max_splits;
    if (splits < 1) splits = 1;
    s.chunk = (uint32_t)((n_right + splits - 1) / splits);
    s.splits = (n_right + s.chunk - 1) / s.chunk;
    return s;
}

cudaError_t launch_stereo_match(const float4* left_kpts, const float4* right_kpts, const uint4* left_desc,
                                const uint4* right_desc, uint32_t* keys, uint32_t* arrivals, uint32_t* tile_counts,
                                StereoMatchRecord* out, uint32_t* count, StereoMatchParams p,
                                const StereoMatchShape& shape, cudaStream_t stream) {
    p.splits = shape.splits;
    p.chunk = shape.chunk;
    match_kernel<<<dim3(shape.left_tiles, shape.splits), kTileLefts, 0, stream>>>(
        left_kpts, right_kpts, left_desc, right_desc, keys, arrivals, tile_counts, p);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    count_launch();
    emit_kernel<<<shape.emit_ctas, kEmitThreads, 0, stream>>>(left_kpts, right_kpts, keys, tile_counts, out,
                                                              count, p, kEmitThreads / kTileLefts);
    e = cudaGetLastError();
    if (e == cudaSuccess) count_launch();
    return e;
}

cudaError_t launch_stereo_match_banded(const float4* left_kpts, const float4* right_kpts, const uint4* left_desc,
                                       const uint4* right_desc, const StereoBandScratch& band, uint32_t* keys,
                                       uint32_t* tile_counts, StereoMatchRecord* out, uint32_t* count,
                                       StereoMatchParams p, int sm_count, cudaStream_t stream) {
    (void)sm_count;
    const uint32_t count_ctas = (p.n_right + kCountThreads - 1) / kCountThreads;
    const uint32_t tiles = (p.n_left + kTileLefts - 1) / kTileLefts;
    bucket_count_kernel<<<count_ctas, kCountThreads, 0, stream>>>(right_kpts, p.n_right, band.hist, band.arrival,
                                                                  band.row_start, band.cursor, tile_counts, tiles);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    count_launch();
    bucket_scatter_kernel<<<(p.n_right + 255) / 256, 256, 0, stream>>>(right_kpts, right_desc, p.n_right,
                                                                       band.cursor, band.pos, band.desc, band.idx);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    count_launch();
    match_banded_kernel<<<(p.n_left + kBandLefts - 1) / kBandLefts, kBandThreads, 0, stream>>>(left_kpts, left_desc, band.row_start, band.pos,
                                                            band.desc, band.idx, keys, tile_counts, p);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    count_launch();
    emit_kernel<<<(p.n_left + kEmitThreads - 1) / kEmitThreads, kEmitThreads, 0, stream>>>(
        left_kpts, right_kpts, keys, tile_counts, out, count, p, kEmitThreads / kTileLefts);
    e = cudaGetLastError();
    if (e == cudaSuccess) count_launch();
    return e;
}

}  // namespace vxsgm
