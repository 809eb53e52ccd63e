// Path aggregation of semi-global matching, across-lanes scan form: one segment
// of lanes per scanline, the disparities of a pixel spread over the segment's
// lanes, the recurrence over d evaluated as a prefix scan with warp shuffles.
// Plans with little work (a single pair, small batches) run this form: every
// scanline gets 8..32 threads instead of one, so a lone pair fills the GPU and
// a pixel step costs a scan of log2(lanes) shuffle rounds instead of a serial
// chain of D dependent steps.
//
// Semantics (vx-vision/shaders/SGMStereo.metal:120-172), per scanline, per
// pixel, for d = 0..D-1 with ONE array Lp[] updated in place (so o1 is this
// pixel's new value at d-1), all values ushort:
//     o0 = Lp[d], o1 = u16(Lnew[d-1] + P1) (0xFFFF at d = 0),
//     o2 = u16(Lp[d+1] + P1) (0xFFFF at d = D-1), o3 = u16(m + P2),
//     Lnew[d] = u16(C + min(o0, o1, o2, o3) - m),   m = min of the previous pixel.
//
// The scan. Written in exact integers, with A_d = min(o0, o2, o3) (all from the
// previous pixel), a_d = C_d - m + A_d and b_d = C_d - m + P1, one pixel is
//     y_d = min(a_d, y_{d-1} + b_d),   y_{-1} = +inf,
// a composition of the maps f_d(x) = min(a_d, x + b_d) of the (min, +)
// semiring, which compose in closed form:
//     (f_2 . f_1)(x) = min(min(a_2, a_1 + b_2), x + (b_1 + b_2)),
// so (a, b) pairs form an associative scan. A lane composes its K consecutive
// disparities serially, the segment scans the lanes' compositions (Kogge-Stone,
// shuffles of width = segment), and each lane then applies the incoming value
// to its K disparities. Pads (d >= D) are identity maps (a = +inf, b = 0), so
// their values copy the last real one and never change a minimum or maximum.
//
// Exactness. The integers equal the shader's ushort values as long as no
// ushort operation of the pixel leaves [0, 65535]. Sufficient, and checked per
// pixel on the whole segment: the previous vector's maximum + P1 <= 65535 (o2),
// m + P2 <= 65535 (o3), and the new vector's minimum >= 0 and maximum + P1 <=
// 65535 (o1 and the result). A pixel that fails the check (the shader's values
// wrapped, which happens where the in-place o1 term pulls a value below m:
// rare with the usual penalties) is recomputed in the shader's own order:
// lane by lane, each lane running its K disparities in ushort arithmetic with
// the previous lane's last value broadcast to it.
//
// Data. Costs come from the pair's byte cost volume (cost.cu; Dv bytes a
// pixel, 64 where x - d < 0), K = 8 bytes a lane (a scanline takes Dv / 8
// lanes: a segment of 2..32), loaded two pixel steps ahead.
// The state of a scanline stays in registers (K values a lane). Results go to
// the same path slabs as the other forms: a byte vector (K bytes a lane, one
// coalesced store a segment) or, for a vector with a value of 255 or more, the
// escape marker in byte 0 (and, with a shadow pool, the slot in bytes 4..7)
// and the exact u16 values in the shadow; wide-slab pairs write every vector
// to the u16 slab.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdio>
#include <cstdlib>

#include "kernels.cuh"
#include "launch.hpp"

namespace vxsgm {
namespace scan {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kInf = 1 << 30;     // above any exact value (|values| < 2^25), no overflow when added to
constexpr int kThreads = 256;

template <int K>
__device__ __forceinline__ void load_costs(const uint8_t* p, bool on, uint32_t (&w)[K / 4]) {
    static_assert(K == 8, "eight disparities a lane");
    const uint2 v = on ? __ldg(reinterpret_cast<const uint2*>(p)) : make_uint2(0u, 0u);
    w[0] = v.x;
    w[1] = v.y;
}

// Cost of disparity j of the lane (byte j of its words).
template <int K>
__device__ __forceinline__ int cost_at(const uint32_t (&w)[K / 4], int j) {
    return (int)__byte_perm(w[j >> 2], 0u, 0x4440u | (uint32_t)(j & 3));
}

// Minimum / maximum over the lanes of a segment (width seg, a power of two).
__device__ __forceinline__ int seg_min(int v, int seg) {
    if (seg == 32) return __reduce_min_sync(kFull, v);
    for (int o = seg >> 1; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(kFull, v, o, seg));
    return v;
}
__device__ __forceinline__ int seg_max(int v, int seg) {
    if (seg == 32) return __reduce_max_sync(kFull, v);
    for (int o = seg >> 1; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(kFull, v, o, seg));
    return v;
}

__device__ __forceinline__ uint32_t pack4(int a, int b, int c, int d) {
    return __byte_perm(__byte_perm((uint32_t)a, (uint32_t)b, 0x0040), __byte_perm((uint32_t)c, (uint32_t)d, 0x0040),
                       0x5410);
}
__device__ __forceinline__ uint32_t pack2(int a, int b) { return __byte_perm((uint32_t)a, (uint32_t)b, 0x5410); }

// One unit: the warp's 32 / seg scanlines first.. of one (pair, path), each on
// one segment of seg lanes; lane li of a segment holds disparities
// d0 = li*K .. d0+K-1 (lanes li >= lanes hold only pads). All lanes run every
// step (the shuffles are warp-collective); a segment outside its scanline's
// steps computes values it never stores.
// NP (no pads): D is a multiple of 16 (D = Dv), so every disparity of a lane
// li < lanes is real, d = D-1 is the last one of lane lanes-1 (its o2 = 0xFFFF
// comes from a next-lane value of 0xFFFF - P1) and only the lanes past `lanes`
// need masking, once per step. Otherwise each disparity is tested.
template <int K, bool CP, bool NP>
__device__ __forceinline__ void run_unit(const PairDev& pr, const JobDev& job, int first, const ScanGeometry g,
                                         int lane) {
    const int W = pr.width, H = pr.height, D = pr.nd, Dv = pr.nd_vec, Dp = pr.nd_pad;
    const int P1 = pr.p1, P2 = pr.p2;
    const bool wide = pr.wide_slabs != 0;
    const int seg = g.seg;
    const int sl = lane / seg, li = lane % seg;
    const int d0 = li * K;
    const bool lane_on = li < g.lanes;
    const bool last_lane = li == g.lanes - 1;
    const int k = first + sl;
    const int dx = job.dx, dy = job.dy;

    // Steps [tb, te) of this scanline and its pixel index base + t * step.
    int tb = INT_MAX, te = -1;
    ptrdiff_t base = 0, step = 0;
    if (k < job.num_scanlines) {
        if (dy == 0) {
            tb = 0;
            te = W;
            base = (ptrdiff_t)k * W + (dx > 0 ? 0 : W - 1);
            step = dx;
        } else {
            const int kk = job.k_min + k;
            if (dx == 0) { tb = 0; te = H; }
            else if (dx > 0) { tb = max(0, -kk); te = min(H, W - kk); }
            else { tb = max(0, kk - W + 1); te = min(H, kk + 1); }
            base = (ptrdiff_t)(dy > 0 ? 0 : H - 1) * W + kk;
            step = (ptrdiff_t)dy * W + dx;
        }
    }
    const int t_lo = __reduce_min_sync(kFull, tb), t_hi = __reduce_max_sync(kFull, te);
    if (t_lo >= t_hi) return;

    const uint8_t* __restrict__ CV = pr.costs;
    auto on_step = [&](int t) { return t >= tb && t < te; };
    auto cost_row = [&](int t) { return on_step(t) ? CV + (size_t)(base + t * step) * Dv + d0 : CV; };
    uint8_t* slab = pr.slabs + pr.slab_stride * (size_t)job.path;
    uint16_t* shadow_path = pr.shadow + pr.shadow_stride * (size_t)job.path;
    const EscapeTarget et = CP ? escape_target(pr, job.path) : EscapeTarget{};
    // A disparity of this lane takes part (NP: every one of an active lane).
    auto real = [&](int j) { return NP ? true : d0 + j < D; };

    int L[K];                 // the scanline's state (previous pixel), disparities d0..d0+K-1
    int m = 0, pmx = 0;       // previous pixel's minimum and maximum
#pragma unroll
    for (int j = 0; j < K; ++j) L[j] = 0;
    uint32_t c0[K / 4], c1[K / 4], c2[K / 4];
    load_costs<K>(cost_row(t_lo), on_step(t_lo) && lane_on, c0);
    load_costs<K>(cost_row(t_lo + 1), on_step(t_lo + 1) && lane_on, c1);

    for (int t = t_lo; t < t_hi; ++t) {
        const bool active = on_step(t);
        load_costs<K>(cost_row(t + 2), on_step(t + 2) && lane_on, c2);   // two steps ahead
        if (__any_sync(kFull, t == tb)) {   // a scanline starts: Lp = 0, m = 0 give L = C (the shader's step 0)
            if (t == tb) {
#pragma unroll
                for (int j = 0; j < K; ++j) L[j] = 0;
                m = 0;
                pmx = 0;
            }
        }
        int Lnext = __shfl_down_sync(kFull, L[0], 1, seg);   // the next lane's Lp[d0 + K]
        if (NP && last_lane) Lnext = 0xFFFF - P1;             // o2 of d = D-1 is 0xFFFF
        const int o3 = m + P2;
        const int p1m = P1 - m;

        // a_d (then y_d in place) and the lane's composition (AL, BL).
        int y[K];
        int AL = kInf, BL = 0;
#pragma unroll
        for (int j = 0; j < K; ++j) {
            const int c = cost_at<K>(c0, j);
            const int nb = j + 1 < K ? L[j + 1] : Lnext;
            int o2 = nb + P1;
            if (!NP && d0 + j == D - 1) o2 = 0xFFFF;
            y[j] = real(j) ? c + __vimin3_s32(L[j], o2, o3) - m : kInf;
            const int b = real(j) ? c + p1m : 0;
            AL = j == 0 ? y[0] : __viaddmin_s32(AL, b, y[j]);
            BL += b;
        }
        // Segment scan of the lanes' maps: lane li gets the composition of lanes 0..li.
        for (int o = 1; o < seg; o <<= 1) {
            const int Ap = __shfl_up_sync(kFull, AL, o, seg);
            const int Bp = __shfl_up_sync(kFull, BL, o, seg);
            if (li >= o) {
                AL = min(AL, Ap + BL);
                BL += Bp;
            }
        }
        int X = __shfl_up_sync(kFull, AL, 1, seg);   // y at d0 - 1
        if (li == 0) X = kInf;
#pragma unroll
        for (int j = 0; j < K; ++j) {
            const int b = real(j) ? cost_at<K>(c0, j) + p1m : 0;
            y[j] = __viaddmin_s32(X, b, y[j]);
            X = y[j];
        }
        int mn = y[0], mx = y[0];
#pragma unroll
        for (int j = 1; j + 1 < K; j += 2) {
            mn = __vimin3_s32(mn, y[j], y[j + 1]);
            mx = __vimax3_s32(mx, y[j], y[j + 1]);
        }
        mn = min(mn, y[K - 1]);
        mx = max(mx, y[K - 1]);
        if (!lane_on) {       // lanes past the vector: identities of the reductions
            mn = INT_MAX;
            mx = INT_MIN;
        }
        mn = seg_min(mn, seg);
        mx = seg_max(mx, seg);
        const bool exact = pmx + P1 <= 0xFFFF && o3 <= 0xFFFF && mn >= 0 && mx + P1 <= 0xFFFF;

        // Pixels whose ushort values wrapped: the shader's serial order, lane by lane.
        if (__any_sync(kFull, active && !exact)) {
            const bool redo = active && !exact;
            int carry = 0;    // Lnew[d0 - 1] of the segment, from the previous lane
            for (int s = 0; s < g.lanes; ++s) {
                if (redo && li == s) {
                    int prev = carry;
#pragma unroll
                    for (int j = 0; j < K; ++j) {
                        const int d = d0 + j;
                        if (d < D) {
                            const int nb = j + 1 < K ? L[j + 1] : Lnext;
                            const int q0 = L[j];
                            const int q1 = d == 0 ? 0xFFFF : ((prev + P1) & 0xFFFF);
                            const int q2 = d == D - 1 ? 0xFFFF : ((nb + P1) & 0xFFFF);
                            const int q3 = (m + P2) & 0xFFFF;
                            prev = (cost_at<K>(c0, j) + min(min(q0, q1), min(q2, q3)) - m) & 0xFFFF;
                        }
                        y[j] = prev;  // pads repeat the last value
                    }
                }
                carry = __shfl_sync(kFull, y[K - 1], s, seg);
            }
            int rmn = INT_MAX, rmx = INT_MIN;
#pragma unroll
            for (int j = 0; j < K; ++j)
                if (lane_on && d0 + j < D) {
                    rmn = min(rmn, y[j]);
                    rmx = max(rmx, y[j]);
                }
            rmn = seg_min(rmn, seg);
            rmx = seg_max(rmx, seg);
            if (redo) {
                mn = rmn;
                mx = rmx;
            }
        }

        // Output of the pixel.
        const size_t pix = active ? (size_t)(base + t * step) : 0;
        const bool esc = !wide && mx >= 0xFF;
        uint32_t slot = kNoSlot;
        if (CP && __any_sync(kFull, active && esc)) {
            if (active && esc && li == 0) slot = take_slot(et, pix);
            slot = __shfl_sync(kFull, slot, 0, seg);
        }
        if (active && lane_on && !wide) {
            uint32_t w[K / 4];
#pragma unroll
            for (int i = 0; i < K / 4; ++i) w[i] = pack4(y[4 * i], y[4 * i + 1], y[4 * i + 2], y[4 * i + 3]);
            if (esc && li == 0) {
                w[0] |= 0xFFu;                        // the escape marker (byte 0)
                if (CP) w[1] = slot;                  // the shadow slot (bytes 4..7)
            }
            uint8_t* row = slab + pix * Dv + d0;
            __stcs(reinterpret_cast<uint2*>(row), make_uint2(w[0], w[1]));
        }
        if (active && (wide || esc) && d0 < Dp) {
            uint16_t* dst = nullptr;
            if (!CP || wide) dst = shadow_path + pix * Dp + d0;
            else if (slot != kNoSlot) dst = et.shadow + (size_t)slot * Dp + d0;
            if (dst) {
                __stcs(reinterpret_cast<uint4*>(dst),
                       make_uint4(pack2(y[0], y[1]), pack2(y[2], y[3]), pack2(y[4], y[5]), pack2(y[6], y[7])));
            }
        }

#pragma unroll
        for (int j = 0; j < K; ++j) L[j] = y[j];
        m = mn;
        pmx = mx;
#pragma unroll
        for (int i = 0; i < K / 4; ++i) {
            c0[i] = c1[i];
            c1[i] = c2[i];
        }
    }
}

template <bool CP>
__global__ void __launch_bounds__(kThreads, 3)
scan_kernel(const PairDev* __restrict__ pairs, const JobDev* __restrict__ jobs, const UnitDev* __restrict__ units,
            const int num_units, unsigned* __restrict__ counter) {
    const int lane = threadIdx.x & 31;
    // First unit of a warp by an interleaved rank (warp w of CTA b: w * grid + b),
    // so that the first, longest units of the LPT order go one to an SM before any
    // SM gets a second; later units come from the counter, after the warps' firsts.
    const int warps = (int)(gridDim.x * (blockDim.x >> 5));
    int u = (int)((threadIdx.x >> 5) * gridDim.x + blockIdx.x);
    for (;;) {
        if (u >= num_units) break;
        const UnitDev unit = units[u];
        const JobDev job = jobs[unit.job];
        const PairDev& pr = pairs[job.pair];
        const ScanGeometry g = scan_geometry(pr.nd_vec);
        if (pr.nd == pr.nd_vec) run_unit<8, CP, true>(pr, job, unit.first_scanline, g, lane);
        else run_unit<8, CP, false>(pr, job, unit.first_scanline, g, lane);
        __syncwarp();
        if (lane == 0) u = warps + (int)atomicAdd(counter, 1u);
        u = __shfl_sync(kFull, u, 0);
    }
}

const void* scan_kernel_fn(bool compact) {
    return compact ? (const void*)scan_kernel<true> : (const void*)scan_kernel<false>;
}

}  // namespace

cudaError_t launch(const PairDev* d_pairs, const JobDev* d_jobs, const UnitDev* d_units, int num_units,
                   unsigned* counter, cudaStream_t stream, bool compact) {
    if (num_units <= 0) return cudaSuccess;
    int dev = 0, sms = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const void* fn = scan_kernel_fn(compact);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kThreads, 0) != cudaSuccess || per_sm < 1) {
        cudaGetLastError();
        per_sm = 1;
    }
    // At least one CTA an SM even for few units: a lone pair's units then run one
    // warp to a scheduler where they can (its scanlines are latency-bound chains).
    int grid = sms * per_sm;
    const int needed = std::max((num_units + kThreads / 32 - 1) / (kThreads / 32), sms);
    if (grid > needed) grid = needed;
    if (std::getenv("VX_SGM_DEBUG"))
        std::fprintf(stderr, "vx_sgm: aggregation (scan) %d CTAs x %d threads (%d an SM), %d units\n", grid, kThreads,
                     per_sm, num_units);
    count_launch();
    void* args[] = {&d_pairs, &d_jobs, &d_units, &num_units, &counter};
    return cudaLaunchKernel(fn, dim3(grid), dim3(kThreads), args, 0, stream);
}

}  // namespace scan
}  // namespace vxsgm
