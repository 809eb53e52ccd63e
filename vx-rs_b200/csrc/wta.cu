// Winner-take-all, parabola subpixel refinement and left-right check, fused
// with the sum of the per-path slabs. One CTA per (pair, image row).
//
// Semantics (vx-vision/shaders/SGMStereo.metal:179-214):
//   S(d)   = sum over paths of L_r(d), modulo 2^16 (the shader's ushort +=)
//   best_d = first minimum of S over d (strict '<' from 0xFFFF)
//   disp   = best_d + (c0 - c2) / (2 (c0 + c2 - 2 c1)) when 0 < best_d < D-1 and
//            the denominator is non-zero, with c0,c1,c2 = S(best_d-1..best_d+1)
//            (IEEE single precision, correctly rounded division).
// Extension: right-view WTA dR(x') = first minimum over d of S(x'+d, d) with
// x'+d < W; a pixel is invalid when x - dL < 0 or |dL - dR(x - dL)| > tol.
// Optional depth output fx*B/disparity for valid pixels with disparity > 0.
//
// Mapping: lanes span disparities (8 per lane: 8 bytes of a byte-slab vector,
// or 16 bytes of a wide one) so slab reads are coalesced; a warp covers 32/seg
// pixels at once. Sums are kept as u16 pairs (d, d+1) in 32-bit words and added
// per half (wrapping modulo 2^16); a byte is widened into its half by a byte
// permute. The loads of all paths of a pixel group are issued before any is
// used (the path count is a template parameter). An escaped byte vector (0xFF
// in byte 0, held by the pixel's first lane) is left out of the byte sum and
// its exact u16 values are read from the shadow slab instead. The
// argmin is a min over the key (S << 8 | d), which orders by cost then by d,
// i.e. the first minimum. The right-view argmin of the row is accumulated in
// shared memory with atomicMin on the same keys.
#include <cuda_runtime.h>

#include "kernels.cuh"
#include "launch.hpp"

namespace vxsgm {

namespace {

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ int find_pair_by_row(const PairDev* pairs, int n, int row) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (pairs[mid].row_begin <= row) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// acc[k] += (d = 2k, d = 2k+1) of 8 byte values (v.x: d 0..3, v.y: d 4..7).
__device__ __forceinline__ void add_bytes(uint32_t (&acc)[4], const uint2 v) {
    acc[0] = __vadd2(acc[0], __byte_perm(v.x, 0u, 0x4140));
    acc[1] = __vadd2(acc[1], __byte_perm(v.x, 0u, 0x4342));
    acc[2] = __vadd2(acc[2], __byte_perm(v.y, 0u, 0x4140));
    acc[3] = __vadd2(acc[3], __byte_perm(v.y, 0u, 0x4342));
}
// The same for 8 u16 values (already (d, d+1) pairs).
__device__ __forceinline__ void add_u16(uint32_t (&acc)[4], const uint4 a) {
    acc[0] = __vadd2(acc[0], a.x);
    acc[1] = __vadd2(acc[1], a.y);
    acc[2] = __vadd2(acc[2], a.z);
    acc[3] = __vadd2(acc[3], a.w);
}

// Sum over the NP paths of the 8 disparities d = 8c..8c+7 of pixel pix (lanes
// with act = false contribute nothing but take part in the warp shuffles).
template <int NP, bool WIDE>
__device__ __forceinline__ void sum_paths(const PairDev& pr, size_t pix, int c, bool act, int lead,
                                          uint32_t (&acc)[4]) {
    const int Dp = pr.nd_pad;
    const bool in_dp = act && 8 * c < Dp;           // lanes past Dp (Dv = Dp + 8) read no shadow
    const uint4 z4 = make_uint4(0u, 0u, 0u, 0u);
    if (WIDE) {
        uint4 v[NP];
#pragma unroll
        for (int p = 0; p < NP; ++p)
            v[p] = in_dp ? __ldcs(reinterpret_cast<const uint4*>(pr.shadow + pr.shadow_stride * p +
                                                                   pix * Dp + 8 * c))
                         : z4;
#pragma unroll
        for (int p = 0; p < NP; ++p) add_u16(acc, v[p]);
        return;
    }
    const int Dv = pr.nd_vec;
    uint2 v[NP];
#pragma unroll
    for (int p = 0; p < NP; ++p)
        v[p] = act ? __ldcs(reinterpret_cast<const uint2*>(pr.slabs + pr.slab_stride * p + pix * Dv + 8 * c))
                   : make_uint2(0u, 0u);
    unsigned esc = 0u;
#pragma unroll
    for (int p = 0; p < NP; ++p) {
        if ((__shfl_sync(kFull, v[p].x, lead) & 0xFFu) == 0xFFu)
            esc |= 1u << p;
        else
            add_bytes(acc, v[p]);
    }
    if (__any_sync(kFull, esc != 0u)) {             // rare: escaped vectors from the shadow
#pragma unroll
        for (int p = 0; p < NP; ++p)
            if (in_dp && ((esc >> p) & 1u))
                add_u16(acc, __ldcs(reinterpret_cast<const uint4*>(pr.shadow + pr.shadow_stride * p +
                                                                     pix * Dp + 8 * c)));
    }
}

// Five CTAs per SM (at most 51 registers a thread) keep enough slab loads in flight.
__global__ void __launch_bounds__(kWtaThreads, 5)
wta_kernel(const PairDev* __restrict__ pairs, int num_pairs) {
    extern __shared__ uint32_t smem[];
    const int pi = find_pair_by_row(pairs, num_pairs, blockIdx.x);
    const PairDev& pr = pairs[pi];
    const int y = blockIdx.x - pr.row_begin;
    const int W = pr.width, D = pr.nd, P = pr.num_paths;
    const bool lr = pr.lr_check != 0;

    uint32_t* right_key = smem;                               // W keys (LR only)
    int* best_d = reinterpret_cast<int*>(smem + W);           // W
    float* disp = reinterpret_cast<float*>(smem + 2 * W);     // W

    if (lr)
        for (int x = threadIdx.x; x < W; x += blockDim.x) right_key[x] = 0xFFFFFFFFu;
    __syncthreads();

    const int chunks = pr.nd_vec / 8;               // 8-disparity chunks per pixel
    int seg = 1;
    while (seg < chunks) seg <<= 1;                 // lanes per pixel (power of two)
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwarps = blockDim.x >> 5;
    const int sub = lane / seg, c = lane % seg;
    const int ppw = 32 / seg;
    const int kind = (P == 2 ? 0 : P == 4 ? 1 : 2) + (pr.wide_slabs ? 3 : 0);

    for (int xb = warp * ppw; xb < W; xb += nwarps * ppw) {
        const int x = xb + sub;
        const bool act = x < W && c < chunks;
        const size_t pix = (size_t)y * W + (act ? x : 0);
        uint32_t acc[4] = {0u, 0u, 0u, 0u};         // acc[k] = S(8c+2k) | S(8c+2k+1) << 16
        switch (kind) {                             // uniform over the CTA
            case 0: sum_paths<2, false>(pr, pix, c, act, sub * seg, acc); break;
            case 1: sum_paths<4, false>(pr, pix, c, act, sub * seg, acc); break;
            case 2: sum_paths<8, false>(pr, pix, c, act, sub * seg, acc); break;
            case 3: sum_paths<2, true>(pr, pix, c, act, sub * seg, acc); break;
            case 4: sum_paths<4, true>(pr, pix, c, act, sub * seg, acc); break;
            default: sum_paths<8, true>(pr, pix, c, act, sub * seg, acc); break;
        }
        uint32_t s[8];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            s[2 * k] = acc[k] & 0xFFFFu;
            s[2 * k + 1] = acc[k] >> 16;
        }
        uint32_t best = 0xFFFFFFFFu;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int d = 8 * c + j;
            if (act && d < D) best = min(best, (s[j] << 8) | (uint32_t)d);
        }
        for (int o = seg >> 1; o > 0; o >>= 1) best = min(best, __shfl_xor_sync(kFull, best, o));
        const int bd = (int)(best & 0xFFu);
        uint32_t c0 = 0, c2 = 0;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int d = 8 * c + j;
            if (act && d == bd - 1) c0 = s[j];
            if (act && d == bd + 1 && d < D) c2 = s[j];
        }
        for (int o = seg >> 1; o > 0; o >>= 1) {
            c0 |= __shfl_xor_sync(kFull, c0, o);
            c2 |= __shfl_xor_sync(kFull, c2, o);
        }
        if (lr && act) {
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int d = 8 * c + j;
                if (d < D && x - d >= 0) atomicMin(&right_key[x - d], (s[j] << 8) | (uint32_t)d);
            }
        }
        if (c == 0 && x < W) {
            float v = (float)bd;
            if (pr.subpixel && bd > 0 && bd < D - 1) {
                const float f0 = (float)c0, f1 = (float)(best >> 8), f2 = (float)c2;
                const float denom = 2.0f * (f0 + f2 - 2.0f * f1);
                if (fabsf(denom) > 1e-6f) v = __fadd_rn(v, __fdiv_rn(f0 - f2, denom));
            }
            best_d[x] = bd;
            disp[x] = v;
        }
    }
    __syncthreads();

    float* out = reinterpret_cast<float*>(reinterpret_cast<char*>(pr.out_f32) + (size_t)y * pr.out_f32_pitch);
    int16_t* out_i = pr.out_i16
        ? reinterpret_cast<int16_t*>(reinterpret_cast<char*>(pr.out_i16) + (size_t)y * pr.out_i16_pitch)
        : nullptr;
    float* out_z = pr.out_depth
        ? reinterpret_cast<float*>(reinterpret_cast<char*>(pr.out_depth) + (size_t)y * pr.out_depth_pitch)
        : nullptr;
    for (int x = threadIdx.x; x < W; x += blockDim.x) {
        const int dl = best_d[x];
        bool valid = true;
        if (lr) {
            const int xr = x - dl;
            valid = xr >= 0 && abs(dl - (int)(right_key[xr] & 0xFFu)) <= pr.lr_tolerance;
        }
        out[x] = valid ? disp[x] : pr.invalid_value;
        if (out_i) out_i[x] = (int16_t)(valid ? dl : -1);
        // Depth epilogue: depth = fx * baseline / disparity (the conversion the
        // reference leaves to its caller, kernels/sgm.rs:284-286).
        if (out_z)
            out_z[x] = (valid && disp[x] > 0.0f) ? __fdiv_rn(pr.depth_scale, disp[x]) : pr.depth_invalid;
    }
}

}  // namespace

size_t wta_smem_bytes(int max_width) { return (size_t)max_width * 3 * sizeof(uint32_t); }

cudaError_t prepare_wta_kernel() {
    return cudaFuncSetAttribute(wta_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)wta_smem_bytes(kMaxWidth));
}

cudaError_t launch_wta(const PairDev* d_pairs, int num_pairs, int total_rows, int max_width,
                       cudaStream_t stream) {
    if (total_rows == 0) return cudaSuccess;
    const size_t smem = wta_smem_bytes(max_width);
    count_launch();
    wta_kernel<<<total_rows, kWtaThreads, smem, stream>>>(d_pairs, num_pairs);
    return cudaGetLastError();
}

}  // namespace vxsgm
