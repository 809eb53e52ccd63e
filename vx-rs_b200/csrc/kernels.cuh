// Device-side descriptors shared by the SGM kernels and their host launchers.
#pragma once
#include <cstddef>
#include <cstdint>

namespace vxsgm {

// One stereo pair of a launch, as the kernels see it. Built on the host by the
// planner (planner.cpp) and copied into the launch's workspace.
struct PairDev {
    const uint8_t* left;   // U8 images, row pitch in bytes
    const uint8_t* right;
    size_t left_pitch, right_pitch;
    void* census_l;        // W*H census words, row-major (y*W + x)
    void* census_r;
    void* census_lt;       // census words in 32-row bands: ((y/32)*W + x)*32 + y%32
    void* census_rt;
    // Per-path costs, pixel-major and d-minor, in one of two formats:
    //  * byte slabs (wide_slabs = 0): num_paths slabs of H*W vectors of Dv bytes.
    //    A vector whose values are all <= 254 is stored as bytes; any other has
    //    byte 0 set to 0xFF (the escape marker), bytes 4..7 set to its slot s
    //    (u32) and its exact u16 values at shadow + s * Dp. With shadow_cap = 0
    //    the shadow holds every vector, s = path * H*W + pixel; otherwise it is
    //    a pool of shadow_cap vectors handed out in escape order by
    //    esc_state[0], and esc_state[1] is set when the pool ran out (the
    //    pair's result is then void and must be recomputed with a full shadow).
    //  * wide slabs (wide_slabs = 1, for configurations whose costs mostly
    //    exceed a byte): every vector in the shadow slabs; no byte slabs.
    uint8_t* slabs;
    size_t slab_stride;    // bytes per slab = H*W*Dv (0 for wide slabs)
    uint16_t* shadow;      // num_paths slabs of H*W*Dp u16
    size_t shadow_stride;  // elements per shadow slab = H*W*Dp
    int wide_slabs;
    uint8_t* costs;        // scanline-pair batches: the matching-cost volume, H*W vectors of Dv bytes
    uint32_t shadow_cap;   // 0: full shadow; else pool size in vectors
    uint32_t* esc_state;   // [0] vectors taken from the pool, [1] overflow flag
    float* out_f32;        // subpixel (or integer) disparity, pitch in bytes
    size_t out_f32_pitch;
    int16_t* out_i16;      // optional integer disparity, pitch in bytes
    size_t out_i16_pitch;
    float* out_depth;      // optional depth fx*B/disparity, pitch in bytes
    size_t out_depth_pitch;
    float depth_scale;     // fx * baseline
    float depth_invalid;   // written where the disparity is invalid or <= 0
    int width, height;
    int nd;                // number of disparities D (1..256)
    int nd_pad;            // Dp = D rounded up to 8
    int nd_vec;            // Dv = D rounded up to 16 (bytes per stored vector)
    int num_paths;
    int p1, p2;            // ushort(p1), ushort(p2)
    int rx, ry;            // census radii
    int subpixel, lr_check, lr_tolerance;
    float invalid_value;
    int census_tile_begin; // first census tile of this pair (census launch)
    int row_begin;         // first cost-volume row of this pair (cost launch)
    // The WTA launch takes the pairs in the order of its row-loop variants (path
    // count, lane form), so that the CTAs running at once mostly share one
    // variant's code: entry k of the pair array also holds the index of the k-th
    // pair of that order and the first WTA row of that k-th pair.
    int wta_pair;
    int wta_row_begin;
};

constexpr uint32_t kNoSlot = 0xFFFFFFFFu;

#ifdef __CUDACC__
// Where the escaped vectors of one path of one pair go, taken from the pair's
// descriptor once per work unit so that the pixel loop keeps it in registers.
struct EscapeTarget {
    uint16_t* shadow;
    uint32_t* esc_state;
    uint32_t cap;        // 0: full shadow
    uint32_t slot_base;  // full shadow: path * H*W
    int Dp;
};

__device__ __forceinline__ EscapeTarget escape_target(const PairDev& pr, int path) {
    return EscapeTarget{pr.shadow, pr.esc_state, pr.shadow_cap,
                        (uint32_t)((size_t)path * pr.width * pr.height), pr.nd_pad};
}

// The shadow slot of an escaped vector at pixel `pix` (one lane), or kNoSlot
// when the pool has run out (the overflow flag is then set).
__device__ __forceinline__ uint32_t take_slot(const EscapeTarget& et, size_t pix) {
    if (et.cap == 0) return et.slot_base + (uint32_t)pix;
    const uint32_t s = atomicAdd(&et.esc_state[0], 1u);
    if (s < et.cap) return s;
    atomicExch(&et.esc_state[1], 1u);
    return kNoSlot;
}
#endif

// One aggregation job: one path direction of one pair.
struct JobDev {
    int pair;
    int path;              // slab index within the pair
    int dx, dy;            // unit step of the path
    int num_scanlines;     // H (horizontal), W (vertical), W+H-1 (diagonal)
    int k_min;             // scanline index offset (diagonals with dx = +1 start at -(H-1))
};

// A warp's unit of aggregation work: kUnitScanlines consecutive scanlines of one job.
struct UnitDev {
    int job;
    int first_scanline;
};

constexpr int kCensusTileW = 32;   // census tile: 32 x 32 pixels of one view a CTA
constexpr int kCensusTileH = 32;
constexpr int kCensusThreadsY = 8; // CTA of 32 x 8 threads, four rows a thread
// Asynchronously staged census rows (interior tiles): the 16-byte aligned
// segment that starts lead = (-rx) mod 16 bytes before x = bx - rx (bx is a
// multiple of 32) and covers the 32 + 2 rx apron columns, rw bytes long.
__host__ __device__ constexpr int census_stage_lead(int rx) { return (16 - (rx & 15)) & 15; }
__host__ __device__ constexpr int census_stage_row_bytes(int rx) {
    return (census_stage_lead(rx) + kCensusTileW + 2 * rx + 15) & ~15;
}
// Dynamic shared memory of a census CTA for radii up to (max_rx, max_ry): the
// clamped staging (rows of 32 + 2 rx bytes) or the asynchronous one (rw bytes).
__host__ __device__ constexpr size_t census_smem_bytes(int max_rx, int max_ry) {
    int w = kCensusTileW + 2 * max_rx;
    for (int rx = 0; rx <= max_rx; ++rx) w = census_stage_row_bytes(rx) > w ? census_stage_row_bytes(rx) : w;
    return (size_t)w * (kCensusTileH + 2 * max_ry);
}
constexpr int kAggWarpsPerBlock = 4;   // warps per TMEM warpgroup
// Scanlines per aggregation work unit of the scanline-pair kernel (one warp:
// two scanlines per lane); the single-scanline kernel takes 32.
constexpr int kUnitScanlines = 64;
// The across-lanes scan form (aggregate_scan.cu): plans select it with this
// value in place of a unit size; its units hold a pair-dependent number of
// scanlines (ScanGeometry::scanlines).
constexpr int kScanForm = 1;
// Geometry of the scan form for a pair with Dv bytes a vector: K = 8
// disparities a lane, `lanes` lanes a scanline in a segment of `seg` lanes (a
// power of two), `scanlines` = 32 / seg scanlines a warp.
struct ScanGeometry {
    int k, lanes, seg, scanlines;
};
__host__ __device__ constexpr ScanGeometry scan_geometry(int nd_vec) {
    const int k = 8;
    const int lanes = nd_vec / k;
    int seg = 1;
    while (seg < lanes) seg <<= 1;
    return ScanGeometry{k, lanes, seg, 32 / seg};
}
// Fewest 64-scanline units for which a batch whose key was not autotuned runs
// the scanline-pair kernel (below: the across-lanes scan kernel; the
// single-scanline kernel is left to the autotuner, which times all three).
constexpr long long kPairKernelMinUnits = 1500;
// Fewer 64-scanline units than this run the across-lanes scan kernel when the
// batch's key was not autotuned (a lone pair, small batches: it gives every
// scanline a segment of lanes, so few scanlines still fill the GPU). Measured
// on B200 with the leading pairs of the 64-pair mixed batch: up to 8 pairs
// (1 020 units) the scan form is fastest (1 pair: 2.29 ms against 6.45 ms for the
// scanline pairs, whose time there is that of its longest unit), from 16 pairs
// (2 232 units) the scanline pairs (6.45 against 9.64 single, 12.0 scan).
constexpr long long kScanFormMaxUnits = 1500;
// Largest aggregation CTA (4 warpgroups); keeps registers per thread <= 128.
constexpr int kAggMaxThreads = 512;
constexpr int kAggMaxWarpgroups = kAggMaxThreads / 128;

// Work queues of one aggregation launch. The units are ordered in classes of
// decreasing padded D, each class longest-first; class c is the range
// [begin[c], begin[c + 1]) of the unit table and has its own counter. Warpgroup
// w keeps its scanlines' state in TMEM columns [col0[w], col0[w] + its budget)
// and pulls units from class first_class[w] (the largest class its budget
// holds) until that is empty, then from the next smaller class, and so on. A
// batch of one D (or any single-class plan) has one queue in plain
// longest-first order.
constexpr int kMaxQueueClasses = 4;
struct AggQueues {
    int n_classes;
    int begin[kMaxQueueClasses + 1];
    int col0[kAggMaxWarpgroups];
    int first_class[kAggMaxWarpgroups];
};
// Guard words before and after every row-major census plane: the aggregation
// kernel stages aligned 16-byte chunks that may extend past the first and last
// row by up to 256 + 72 words.
constexpr int kCensusGuardWords = 352;

// Shared memory of one aggregation warp (scanline-pair form) for a batch whose
// largest padded D is dp_max: the output tile of its 64 scanlines. Tile rows
// hold byte vectors (Dv bytes plus 8, so that the rows' 8-byte stores fall on
// distinct banks) or, when the batch has wide-slab pairs, u16 vectors (2*Dp
// bytes plus 16).
__host__ __device__ constexpr int aggregate_row_bytes(int dp_max, bool wide_tiles) {
    return wide_tiles ? 2 * dp_max + 16 : (dp_max + 15) / 16 * 16 + 8;
}
__host__ __device__ constexpr size_t aggregate_warp_smem(int dp_max, bool wide_tiles) {
    return (size_t)kUnitScanlines * aggregate_row_bytes(dp_max, wide_tiles);
}
__host__ __device__ constexpr size_t aggregate_tile_offset(int dp_max) { return (size_t)(dp_max + 72) * 8; }

constexpr int kWtaThreads = 256;
// Row-loop forms of the WTA kernel: byte slabs summed 16 disparities a lane (a
// pixel's lanes read its whole vector of a path in one round) or 8 a lane, and
// wide slabs (8 u16 a lane). Byte slabs take 16 unless 8 keeps more lanes busy:
// lanes per pixel are a power of two, so Dv / 16 = 9..12 chunks (D = 192: 12 of
// 16 lanes) fill 8 lanes over 3 rounds better.
constexpr int kFormBytes16 = 0, kFormBytes8 = 1, kFormWide = 2;
__host__ __device__ constexpr int wta_disparities_per_lane(int form) { return form == kFormBytes16 ? 16 : 8; }
// Lanes per pixel: the pixel's chunks rounded up to a power of two, at most
// 16 (16-disparity chunks) or 8 (8-disparity chunks).
__host__ __device__ constexpr int wta_lanes_per_pixel(int nd_vec, int form) {
    const int chunks = nd_vec / wta_disparities_per_lane(form);
    const int cap = form == kFormBytes16 ? 16 : 8;
    int seg = 1;
    while (seg < chunks && seg < cap) seg <<= 1;
    return seg;
}
__host__ __device__ constexpr int wta_form(int nd_vec, bool wide) {
    if (wide) return kFormWide;
    // busy lane-rounds per lane-round: chunks / (seg * rounds), compared exactly
    const int c16 = nd_vec / 16, s16 = wta_lanes_per_pixel(nd_vec, kFormBytes16);
    const int c8 = nd_vec / 8, s8 = wta_lanes_per_pixel(nd_vec, kFormBytes8);
    const int slots16 = s16 * ((c16 + s16 - 1) / s16), slots8 = s8 * ((c8 + s8 - 1) / s8);
    return c8 * slots16 > c16 * slots8 ? kFormBytes8 : kFormBytes16;
}
// The row-loop variant of a pair (0..8): path class x form.
__host__ __device__ constexpr int wta_variant(int num_paths, int nd_vec, bool wide) {
    return (num_paths == 2 ? 0 : num_paths == 4 ? 1 : 2) * 3 + wta_form(nd_vec, wide);
}
// u16 sums per WTA warp in shared memory: its pixels (32 / lanes per pixel) x
// their padded disparities (disparities a lane x lanes per pixel x rounds):
// byte slabs 32 x 16 x 1, wide slabs 32 x 8 x 4 at most.
constexpr int kWtaSumsPerWarp = 1024;
// Widest image the WTA kernel accepts (three 4-byte words per pixel and the
// right-view keys' padding, a quarter word per pixel, in shared memory).
constexpr int kMaxWidth = 16384;

}  // namespace vxsgm
