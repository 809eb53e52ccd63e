// Path aggregation of semi-global matching, all paths of all pairs of a batch
// in one persistent launch per kernel variant.
//
// Semantics (vx-vision/shaders/SGMStereo.metal:72-173), per scanline, per pixel,
// for d = 0..D-1 in increasing order with ONE array Lp[] updated in place:
//     C    = popcount(cl(x,y) ^ cr(x-d,y)), or 64 when x-d < 0      (:131-142)
//     o0   = Lp[d]                     (previous pixel)
//     o1   = u16(Lp[d-1] + P1)         (d-1 already rewritten: THIS pixel), 0xFFFF at d=0
//     o2   = u16(Lp[d+1] + P1)         (previous pixel), 0xFFFF at d=D-1
//     o3   = u16(m + P2)               (m = min of the previous pixel)
//     Lp[d]= u16(C + min(o0,o1,o2,o3) - m)                               (:150-161)
// The first pixel of a scanline starts from Lp = 0, m = 0, which makes every
// option >= 0 and the result exactly C, as the shader's step-0 branch does.
// The shader only runs directions (1,0) and (0,1) (sgm.rs:197-200); the other
// six directions are the same recurrence on the other scanline families.
//
// Mapping: one thread owns one scanline and keeps its D costs in registers as
// packed u16 pairs, so the in-place recurrence is a register sweep with no
// cross-lane traffic. A warp takes 32 neighbouring scanlines of one job, laid
// out so that at every step its lanes sit on consecutive pixels of one row
// (vertical, diagonal) or one column (horizontal, which reads the
// column-major census): census loads of a warp are consecutive words.
// Each pixel's D results go to this path's slab with 16-byte stores.
#include <cuda_runtime.h>

#include "kernels.cuh"
#include "launch.hpp"

namespace vxsgm {

namespace {

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ uint32_t popc_xor(uint32_t a, uint32_t b) { return __popc(a ^ b); }
__device__ __forceinline__ uint32_t popc_xor(uint64_t a, uint64_t b) { return __popcll(a ^ b); }

template <int DMAX, bool EXACT, typename CT, bool HORIZ>
__global__ void __launch_bounds__(kAggWarpsPerBlock * 32)
aggregate_kernel(const PairDev* __restrict__ pairs, const JobDev* __restrict__ jobs,
                 const UnitDev* __restrict__ units, int num_units, unsigned* __restrict__ counter) {
    constexpr int NW = DMAX / 2;  // packed u16 pairs per thread
    static_assert(NW % 4 == 0, "DMAX must be a multiple of 8");
    const int lane = threadIdx.x & 31;

    for (;;) {
        int u = 0;
        if (lane == 0) u = (int)atomicAdd(counter, 1u);
        u = __shfl_sync(kFull, u, 0);
        if (u >= num_units) break;

        const UnitDev unit = units[u];
        const JobDev job = jobs[unit.job];
        const PairDev& pr = pairs[job.pair];
        const int W = pr.width, H = pr.height;
        const int D = EXACT ? DMAX : pr.nd;
        const int Dp = pr.nd_pad;
        const uint32_t P1 = (uint32_t)pr.p1, P2 = (uint32_t)pr.p2;
        const int dx = job.dx, dy = job.dy;

        const int i = unit.first_scanline + lane;
        const bool lane_valid = i < job.num_scanlines;
        const int k = job.k_min + i;

        // Pixel of scanline k at step t: (x0 + kx*k + tx*t, y0 + ky*k + ty*t).
        int x0, y0, kx, ky;
        if (dy == 0) { x0 = dx > 0 ? 0 : W - 1; y0 = 0; kx = 0; ky = 1; }
        else { x0 = 0; y0 = dy > 0 ? 0 : H - 1; kx = 1; ky = 0; }
        const int tx = dx, ty = dy;
        int tb, te;
        if (dy == 0) { tb = 0; te = W; }
        else if (dx == 0) { tb = 0; te = H; }
        else if (dx > 0) { tb = max(0, -k); te = min(H, W - k); }
        else { tb = max(0, k - W + 1); te = min(H, k + 1); }
        if (!lane_valid) { tb = 0x7fffffff; te = -1; }
        const int t_lo = __reduce_min_sync(kFull, tb);
        const int t_hi = __reduce_max_sync(kFull, te);

        const CT* __restrict__ CL = static_cast<const CT*>(HORIZ ? pr.census_lt : pr.census_l);
        const CT* __restrict__ CR = static_cast<const CT*>(HORIZ ? pr.census_rt : pr.census_r);
        uint16_t* __restrict__ out = pr.slabs + pr.slab_stride * (size_t)job.path;

        uint32_t Lp[NW];
#pragma unroll
        for (int w = 0; w < NW; ++w) Lp[w] = 0u;
        uint32_t m = 0u;

        for (int t = t_lo; t < t_hi; ++t) {
            if (t < tb || t >= te) continue;
            const int x = x0 + kx * k + tx * t;
            const int y = y0 + ky * k + ty * t;
            CT lc;
            const CT* rp;  // right census of (x, y); (x - d, y) is rp - d*stride
            if (HORIZ) {
                lc = CL[(size_t)x * H + y];
                rp = CR + (size_t)x * H + y;
            } else {
                lc = CL[(size_t)y * W + x];
                rp = CR + (size_t)y * W + x;
            }
            const uint32_t o3 = (m + P2) & 0xFFFFu;
            uint32_t e = 0u, nm = 0xFFFFu;
            uint16_t* dst = out + ((size_t)y * W + x) * Dp;
#pragma unroll
            for (int w = 0; w < NW; w += 4) {
                uint32_t packed[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int wi = w + j;
                    const uint32_t cur = Lp[wi];
                    const uint32_t nxt = (wi + 1 < NW) ? Lp[wi + 1] : 0u;
                    uint32_t ev[2];
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const int d = 2 * wi + h;
                        uint32_t c = 64u;
                        if (x - d >= 0) c = popc_xor(lc, HORIZ ? rp[-(ptrdiff_t)d * H] : rp[-d]);
                        const uint32_t o0 = h ? (cur >> 16) : (cur & 0xFFFFu);
                        const uint32_t nb = h ? (nxt & 0xFFFFu) : (cur >> 16);
                        uint32_t o2 = (nb + P1) & 0xFFFFu;
                        if (EXACT ? (d == DMAX - 1) : (d >= D - 1)) o2 = 0xFFFFu;
                        const uint32_t o1 = (d == 0) ? 0xFFFFu : ((e + P1) & 0xFFFFu);
                        const uint32_t best = min(min(o0, o1), min(o2, o3));
                        e = (c + best - m) & 0xFFFFu;
                        if (EXACT || d < D) nm = min(nm, e);
                        ev[h] = e;
                    }
                    packed[j] = ev[0] | (ev[1] << 16);
                    Lp[wi] = packed[j];
                }
                if (EXACT || 2 * w < D)
                    *reinterpret_cast<uint4*>(dst + 2 * w) =
                        make_uint4(packed[0], packed[1], packed[2], packed[3]);
            }
            m = nm;
        }
    }
}

using AggKernelFn = void (*)(const PairDev*, const JobDev*, const UnitDev*, int, unsigned*);

template <int DMAX, bool EXACT>
AggKernelFn pick_ct_dir(bool census64, bool horizontal) {
    if (census64)
        return horizontal ? aggregate_kernel<DMAX, EXACT, uint64_t, true>
                          : aggregate_kernel<DMAX, EXACT, uint64_t, false>;
    return horizontal ? aggregate_kernel<DMAX, EXACT, uint32_t, true>
                      : aggregate_kernel<DMAX, EXACT, uint32_t, false>;
}

AggKernelFn pick_kernel(const AggVariant& v) {
    if (v.exact) {
        switch (v.dmax) {
            case 64: return pick_ct_dir<64, true>(v.census64, v.horizontal);
            case 128: return pick_ct_dir<128, true>(v.census64, v.horizontal);
            case 192: return pick_ct_dir<192, true>(v.census64, v.horizontal);
            case 256: return pick_ct_dir<256, true>(v.census64, v.horizontal);
        }
    } else {
        switch (v.dmax) {
            case 64: return pick_ct_dir<64, false>(v.census64, v.horizontal);
            case 128: return pick_ct_dir<128, false>(v.census64, v.horizontal);
            case 256: return pick_ct_dir<256, false>(v.census64, v.horizontal);
        }
    }
    return nullptr;
}

}  // namespace

int aggregate_grid_ctas(const AggVariant& v) {
    AggKernelFn fn = pick_kernel(v);
    if (!fn) return 0;
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kAggWarpsPerBlock * 32, 0);
    return sms * (per_sm > 0 ? per_sm : 1);
}

cudaError_t launch_aggregate(const AggVariant& v, const PairDev* d_pairs, const JobDev* d_jobs,
                             const UnitDev* d_units, int num_units, unsigned* counter,
                             int grid_ctas, cudaStream_t stream) {
    if (num_units <= 0) return cudaSuccess;
    AggKernelFn fn = pick_kernel(v);
    if (!fn) return cudaErrorInvalidValue;
    if (grid_ctas <= 0) grid_ctas = aggregate_grid_ctas(v);
    const int needed = (num_units + kAggWarpsPerBlock - 1) / kAggWarpsPerBlock;
    if (grid_ctas > needed) grid_ctas = needed;
    count_launch();
    fn<<<grid_ctas, kAggWarpsPerBlock * 32, 0, stream>>>(d_pairs, d_jobs, d_units, num_units,
                                                         counter);
    return cudaGetLastError();
}

}  // namespace vxsgm
