// Host driver for the literal reference SGM shader ("tier 1" oracle).
//
// TEST INFRASTRUCTURE ONLY. oracle/Makefile compiles vx-vision's
// shaders/SGMStereo.metal unmodified as C++ (through oracle/ref_shim) and links
// it with this file into oracle/_ref/libsgm_ref.so. The entry point below
// replays what vx-vision/src/kernels/sgm.rs:108-265 (SGMStereo::compute_disparity)
// encodes on the GPU: census(left), census(right), aggregation along (1,0) then
// (0,1), WTA. Each Metal thread id becomes one call of the kernel function.
// Scanlines of one aggregation dispatch write disjoint pixels, so they are
// spread over host threads exactly as the GPU spreads them over SIMD lanes.
#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include <metal_stdlib>
using namespace metal;

// Must match vx-vision/shaders/SGMStereo.metal:9-19 field for field.
struct SGMParams {
    uint width;
    uint height;
    uint num_disparities;
    float p1;
    float p2;
    uint census_radius_x;
    uint census_radius_y;
    uint direction_x;
    int direction_y;
};

extern "C" void sgm_census_transform(texture2d<float, access::read> image, uint2* census,
                                     const SGMParams& params, uint2 gid);
extern "C" void sgm_cost_aggregate(uint2* left_census, uint2* right_census, ushort* cost_volume,
                                   const SGMParams& params, uint tid);
extern "C" void sgm_wta_disparity(ushort* cost_volume, texture2d<float, access::write> output,
                                  const SGMParams& params, uint2 gid);

template <typename F>
static void parallel_for(uint n, int nthreads, F f) {
    if (nthreads <= 0) nthreads = (int)std::max(1u, std::thread::hardware_concurrency());
    nthreads = (int)std::min<uint>((uint)nthreads, std::max(1u, n));
    std::atomic<uint> next{0};
    auto body = [&]() {
        for (;;) {
            uint i = next.fetch_add(1);
            if (i >= n) break;
            f(i);
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nthreads; ++t) pool.emplace_back(body);
    body();
    for (auto& t : pool) t.join();
}

extern "C" {

// Runs the reference pipeline on one rectified pair (row pitch == width).
//   census_l / census_r : out, 2 words per pixel (the shader's uint2), nullable
//   cost_volume         : out, W*H*D u16 (HWD order), nullable
//   disparity           : out, W*H f32
// Returns 0, or -1 on bad arguments.
int ref_sgm_compute(const uint8_t* left, const uint8_t* right, int w, int h, int nd, float p1,
                    float p2, int rx, int ry, uint32_t* census_l, uint32_t* census_r,
                    uint16_t* cost_volume, float* disparity, int nthreads) {
    if (w <= 0 || h <= 0 || nd <= 0 || nd > 256 || !left || !right || !disparity) return -1;
    const size_t npx = (size_t)w * h;
    std::vector<uint2> cl(npx), cr(npx);
    std::vector<ushort> cv(npx * (size_t)nd, 0);  // sgm.rs:127-129 zeroes the volume

    SGMParams prm{};
    prm.width = (uint)w;
    prm.height = (uint)h;
    prm.num_disparities = (uint)nd;
    prm.p1 = p1;
    prm.p2 = p2;
    prm.census_radius_x = (uint)rx;
    prm.census_radius_y = (uint)ry;

    texture2d<float, access::read> tl, tr;
    tl.u8 = left;
    tl.width = tl.pitch = (uint)w;
    tr.u8 = right;
    tr.width = tr.pitch = (uint)w;
    parallel_for((uint)h, nthreads, [&](uint y) {
        for (uint x = 0; x < (uint)w; ++x) {
            sgm_census_transform(tl, cl.data(), prm, uint2(x, y));
            sgm_census_transform(tr, cr.data(), prm, uint2(x, y));
        }
    });

    // sgm.rs:197-200: horizontal (1,0) over H rows, then vertical (0,1) over W columns.
    SGMParams ph = prm;
    ph.direction_x = 1;
    ph.direction_y = 0;
    parallel_for((uint)h, nthreads,
                 [&](uint t) { sgm_cost_aggregate(cl.data(), cr.data(), cv.data(), ph, t); });
    SGMParams pv = prm;
    pv.direction_x = 0;
    pv.direction_y = 1;
    parallel_for((uint)w, nthreads,
                 [&](uint t) { sgm_cost_aggregate(cl.data(), cr.data(), cv.data(), pv, t); });

    texture2d<float, access::write> out;
    out.f32 = disparity;
    out.width = out.pitch = (uint)w;
    parallel_for((uint)h, nthreads, [&](uint y) {
        for (uint x = 0; x < (uint)w; ++x) sgm_wta_disparity(cv.data(), out, prm, uint2(x, y));
    });

    if (census_l) std::memcpy(census_l, cl.data(), npx * sizeof(uint2));
    if (census_r) std::memcpy(census_r, cr.data(), npx * sizeof(uint2));
    if (cost_volume) std::memcpy(cost_volume, cv.data(), cv.size() * sizeof(ushort));
    return 0;
}

// Runs one aggregation dispatch of the reference shader for an arbitrary
// direction (dx, dy), accumulating into cost_volume (W*H*D u16, caller-zeroed).
// The shader itself returns early for diagonal directions
// (SGMStereo.metal:100-104); this entry exposes exactly that behaviour.
int ref_sgm_aggregate(const uint32_t* census_l, const uint32_t* census_r, int w, int h, int nd,
                      float p1, float p2, int dx, int dy, uint16_t* cost_volume, int nthreads) {
    if (w <= 0 || h <= 0 || nd <= 0 || nd > 256) return -1;
    SGMParams prm{};
    prm.width = (uint)w;
    prm.height = (uint)h;
    prm.num_disparities = (uint)nd;
    prm.p1 = p1;
    prm.p2 = p2;
    prm.direction_x = (uint)dx;  // SGMParams.direction_x is u32 (types.rs:460)
    prm.direction_y = dy;
    uint n = (dy == 0) ? (uint)h : (uint)w;
    uint2* cl = (uint2*)census_l;
    uint2* cr = (uint2*)census_r;
    parallel_for(n, nthreads, [&](uint t) { sgm_cost_aggregate(cl, cr, cost_volume, prm, t); });
    return 0;
}

}  // extern "C"
