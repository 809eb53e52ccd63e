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
// Mapping: lanes span disparities (16 per lane: 16 bytes of a byte-slab
// vector, so a pixel's lanes read its whole vector of each path in one round;
// 8 per lane of a wide one) so slab reads are coalesced; a warp covers 32/seg
// pixels at once. Sums are kept as u16 pairs in 32-bit words (wide slabs: added
// per half, wrapping modulo 2^16; byte slabs: bytes widened by a mask or a byte
// permute and summed as whole words, see sum_paths). The loads of all paths of
// a pixel group are issued before any is used (the path count is a template
// parameter). An escaped byte vector (0xFF in byte 0, held by the pixel's first
// lane) is taken out of the byte sum and its exact u16 values are read from
// the shadow slab instead. The argmin is a min over the key (S << 8 | d), which
// orders by cost then by d, i.e. the first minimum; S(bd-1) and S(bd+1) for the
// subpixel step come from the lanes that hold them. The right-view argmin of
// the row is accumulated in shared memory with atomicMin on the same keys.
#include <cuda_runtime.h>

#include "kernels.cuh"
#include "launch.hpp"

namespace vxsgm {

namespace {

constexpr unsigned kFull = 0xffffffffu;

// Position k of the WTA order whose rows hold this row (wta_row_begin rises with k).
__device__ __forceinline__ int find_wta_position(const PairDev* pairs, int n, int row) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (pairs[mid].wta_row_begin <= row) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// Per-lane view of one pair, held in registers for the row loop.
struct RowView {
    const uint8_t* slabs;
    const uint16_t* shadow;
    size_t slab_stride, shadow_stride;
    int Dp, Dv;
    uint32_t shadow_cap;  // 0: full shadow; else the pool size (slots beyond it were never written)
};

// The same sums for 8 u16 values (natural (d, d+1) pairs) into lo/hi words
// that hold (d, d+2) pairs: lo0 = (0, 2), hi0 = (1, 3), lo1 = (4, 6), hi1 = (5, 7).
__device__ __forceinline__ void add_u16_split(uint32_t* a, const uint4 v) {
    a[0] = __vadd2(a[0], __byte_perm(v.x, v.y, 0x5410));
    a[1] = __vadd2(a[1], __byte_perm(v.x, v.y, 0x7632));
    a[2] = __vadd2(a[2], __byte_perm(v.z, v.w, 0x5410));
    a[3] = __vadd2(a[3], __byte_perm(v.z, v.w, 0x7632));
}

// Sum over the NP paths of the 8 disparities d = 8c..8c+7 of pixel pix, as
// natural pairs acc[k] = S(8c+2k) | S(8c+2k+1) << 16 (lanes with act = false
// contribute nothing but take part in the warp shuffles).
//
// Byte slabs: a non-escaped byte is at most 254, so 8 of them sum to less than
// 2^11 and whole 32-bit words can be added: the byte pairs (0, 2) and (1, 3) of
// a 4-byte word are widened by a mask and a byte permute and summed with plain
// 3-input adds, no carry reaching the next half. Escaped vectors (marker in the
// byte 0 of the pixel's lane c = 0, shadow slot in its bytes 4..7) are taken
// out again and replaced by their exact u16 values from the shadow with
// per-half wrapping adds (rare).
template <int NP, bool WIDE, bool FIRST>
__device__ __forceinline__ void sum_paths(const RowView& rv, size_t pix, int c, bool act, int lead,
                                          unsigned& em, uint32_t (&acc)[4]) {
    const bool in_dp = act && 8 * c < rv.Dp;        // lanes past Dp (Dv = Dp + 8) read no shadow
    const uint4 z4 = make_uint4(0u, 0u, 0u, 0u);
    if (WIDE) {
        const uint16_t* base = rv.shadow + pix * rv.Dp + 8 * c;
        uint4 v[NP];
#pragma unroll
        for (int p = 0; p < NP; ++p)
            v[p] = in_dp ? __ldcs(reinterpret_cast<const uint4*>(base + rv.shadow_stride * p)) : z4;
#pragma unroll
        for (int p = 0; p < NP; ++p) {
            acc[0] = __vadd2(acc[0], v[p].x);
            acc[1] = __vadd2(acc[1], v[p].y);
            acc[2] = __vadd2(acc[2], v[p].z);
            acc[3] = __vadd2(acc[3], v[p].w);
        }
        return;
    }
    const uint8_t* base = rv.slabs + pix * rv.Dv + 8 * c;
    uint2 v[NP];
#pragma unroll
    for (int p = 0; p < NP; ++p)
        v[p] = act ? __ldg(reinterpret_cast<const uint2*>(base + rv.slab_stride * p)) : make_uint2(0u, 0u);
    constexpr uint32_t M = 0x00FF00FFu;
    uint32_t a[4] = {0u, 0u, 0u, 0u};               // (0,2) (1,3) (4,6) (5,7)
#pragma unroll
    for (int p = 0; p < NP; p += 2) {
        a[0] += (v[p].x & M) + (v[p + 1].x & M);
        a[1] += __byte_perm(v[p].x, 0u, 0x4341) + __byte_perm(v[p + 1].x, 0u, 0x4341);
        a[2] += (v[p].y & M) + (v[p + 1].y & M);
        a[3] += __byte_perm(v[p].y, 0u, 0x4341) + __byte_perm(v[p + 1].y, 0u, 0x4341);
    }
    // Any marker among the paths: their bytes 0 gathered four to a word (byte
    // permutes); a byte 0xFF is a zero byte of the complement, which the
    // borrow test (~g - 0x01..01) & g & 0x80..80 finds exactly. Only the
    // pixel's lane c = 0 holds markers; exact per-path flags are formed in the
    // rare branch.
    uint32_t ff = 0u;
#pragma unroll
    for (int p = 0; p < (FIRST ? NP : 0); p += 4) {
        uint32_t g;
        if (NP == 2) {
            g = __byte_perm(v[p].x, v[p + 1].x, 0x4040);
        } else {
            g = __byte_perm(__byte_perm(v[p].x, v[p + 1].x, 0x0040), __byte_perm(v[p + 2].x, v[p + 3].x, 0x0040),
                            0x5410);
        }
        ff |= (~g - 0x01010101u) & g & 0x80808080u;
    }
    if (FIRST) {                                    // round 0: the lanes c = 0 hold chunk 0
        em = 0u;
        if (__any_sync(kFull, c == 0 && ff != 0u)) {
            unsigned e = 0u;
#pragma unroll
            for (int p = 0; p < NP; ++p) e |= ((v[p].x & 0xFFu) == 0xFFu ? 1u : 0u) << p;
            em = __shfl_sync(kFull, e, lead);       // the pixel's markers (its lane c = 0)
        }
    }
    if (__any_sync(kFull, em != 0u)) {
        // Every escaped byte vector out first (plain subtractions are exact only
        // while no half has wrapped), then the shadow values in.
#pragma unroll
        for (int p = 0; p < NP; ++p) {
            if (act && ((em >> p) & 1u)) {
                a[0] -= v[p].x & M;
                a[1] -= __byte_perm(v[p].x, 0u, 0x4341);
                a[2] -= v[p].y & M;
                a[3] -= __byte_perm(v[p].y, 0u, 0x4341);
            }
        }
        // The slot: with a full shadow the vector's own place (path, pixel);
        // with a pool the one written into the row's bytes 4..7.
        const uint8_t* row0 = rv.slabs + pix * rv.Dv;  // the pixel's rows start here in every slab
#pragma unroll
        for (int p = 0; p < NP; ++p) {
            if (in_dp && ((em >> p) & 1u)) {
                const uint16_t* src = rv.shadow + rv.shadow_stride * p + pix * rv.Dp;
                bool ok = true;
                if (rv.shadow_cap != 0) {
                    const uint32_t slot = *reinterpret_cast<const uint32_t*>(row0 + rv.slab_stride * p + 4);
                    ok = slot < rv.shadow_cap;
                    src = rv.shadow + (size_t)slot * rv.Dp;
                }
                if (ok) add_u16_split(a, __ldcs(reinterpret_cast<const uint4*>(src + 8 * c)));
            }
        }
    }
    acc[0] = __byte_perm(a[0], a[1], 0x5410);
    acc[1] = __byte_perm(a[0], a[1], 0x7632);
    acc[2] = __byte_perm(a[2], a[3], 0x5410);
    acc[3] = __byte_perm(a[2], a[3], 0x7632);
}

// Byte slabs, 16 disparities a lane: the sums S(16c .. 16c+15) of pixel pix as
// natural pairs acc[k] = S(16c+2k) | S(16c+2k+1) << 16 from one 16-byte load
// per path, so a pixel's vector (Dv <= 256 bytes) is read by its lanes in one
// round of whole lines. Bytes are widened and summed as whole words as in
// sum_paths. Escaped vectors are taken out and their shadow values put in with
// per-half wrapping arithmetic (exact modulo 2^16 in any order); the byte
// vector is read again there (rare), so the loads need not stay live.
template <int NP, bool FIRST>
__device__ __forceinline__ void sum_bytes16(const RowView& rv, size_t pix, int c, bool act, int lead,
                                            unsigned& em, uint32_t (&acc)[8]) {
    constexpr uint32_t M = 0x00FF00FFu;
    const uint8_t* base = rv.slabs + pix * rv.Dv + 16 * c;
    uint4 v[NP];
#pragma unroll
    for (int p = 0; p < NP; ++p)
        v[p] = act ? __ldg(reinterpret_cast<const uint4*>(base + rv.slab_stride * p)) : make_uint4(0u, 0u, 0u, 0u);
    uint32_t a[8] = {0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u};   // word i: (4i, 4i+2) in a[2i], (4i+1, 4i+3) in a[2i+1]
#pragma unroll
    for (int p = 0; p < NP; p += 2) {
        a[0] += (v[p].x & M) + (v[p + 1].x & M);
        a[1] += __byte_perm(v[p].x, 0u, 0x4341) + __byte_perm(v[p + 1].x, 0u, 0x4341);
        a[2] += (v[p].y & M) + (v[p + 1].y & M);
        a[3] += __byte_perm(v[p].y, 0u, 0x4341) + __byte_perm(v[p + 1].y, 0u, 0x4341);
        a[4] += (v[p].z & M) + (v[p + 1].z & M);
        a[5] += __byte_perm(v[p].z, 0u, 0x4341) + __byte_perm(v[p + 1].z, 0u, 0x4341);
        a[6] += (v[p].w & M) + (v[p + 1].w & M);
        a[7] += __byte_perm(v[p].w, 0u, 0x4341) + __byte_perm(v[p + 1].w, 0u, 0x4341);
    }
    if (FIRST) {                                    // the markers: bytes 0 of the pixel's lane c = 0
        uint32_t ff = 0u;
#pragma unroll
        for (int p = 0; p < NP; p += 4) {
            uint32_t g;
            if (NP == 2) {
                g = __byte_perm(v[p].x, v[p + 1].x, 0x4040);
            } else {
                g = __byte_perm(__byte_perm(v[p].x, v[p + 1].x, 0x0040),
                                __byte_perm(v[p + 2].x, v[p + 3].x, 0x0040), 0x5410);
            }
            ff |= (~g - 0x01010101u) & g & 0x80808080u;
        }
        em = 0u;
        if (__any_sync(kFull, c == 0 && ff != 0u)) {
            unsigned e = 0u;
#pragma unroll
            for (int p = 0; p < NP; ++p) e |= ((v[p].x & 0xFFu) == 0xFFu ? 1u : 0u) << p;
            em = __shfl_sync(kFull, e, lead);
        }
    }
    if (__any_sync(kFull, em != 0u)) {
        const uint8_t* row0 = rv.slabs + pix * rv.Dv;
#pragma unroll
        for (int p = 0; p < NP; ++p) {
            if (!act || !((em >> p) & 1u)) continue;
            const uint4 b = __ldg(reinterpret_cast<const uint4*>(base + rv.slab_stride * p));
            a[0] = __vsub2(a[0], b.x & M);
            a[1] = __vsub2(a[1], __byte_perm(b.x, 0u, 0x4341));
            a[2] = __vsub2(a[2], b.y & M);
            a[3] = __vsub2(a[3], __byte_perm(b.y, 0u, 0x4341));
            a[4] = __vsub2(a[4], b.z & M);
            a[5] = __vsub2(a[5], __byte_perm(b.z, 0u, 0x4341));
            a[6] = __vsub2(a[6], b.w & M);
            a[7] = __vsub2(a[7], __byte_perm(b.w, 0u, 0x4341));
            const uint16_t* src = rv.shadow + rv.shadow_stride * p + pix * rv.Dp;
            if (rv.shadow_cap != 0) {
                const uint32_t slot = *reinterpret_cast<const uint32_t*>(row0 + rv.slab_stride * p + 4);
                if (slot >= rv.shadow_cap) continue;
                src = rv.shadow + (size_t)slot * rv.Dp;
            }
            // Lanes past Dp read no shadow (Dv can be Dp + 8).
            if (16 * c < rv.Dp) add_u16_split(a, __ldcs(reinterpret_cast<const uint4*>(src + 16 * c)));
            if (16 * c + 8 < rv.Dp) add_u16_split(a + 4, __ldcs(reinterpret_cast<const uint4*>(src + 16 * c + 8)));
        }
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        acc[2 * i] = __byte_perm(a[2 * i], a[2 * i + 1], 0x5410);
        acc[2 * i + 1] = __byte_perm(a[2 * i], a[2 * i + 1], 0x7632);
    }
}

// Right-view keys in shared memory: column a at a + (a / 16) * pad. A warp's
// atomicMin of one key index j goes to columns x + s - K c - j (s its pixel,
// c the lane in the pixel), K c apart across lanes: unpadded, the 16-disparity
// lanes of a byte slab fall on 2 banks a pixel (6- to 8-way conflicts at 16
// lanes a pixel, 4-way at 8). pad = 2 words per 16 at 16 lanes a pixel and 4
// at 8 spread them over all 32 banks; at fewer lanes a pixel, and for the
// 8-disparity forms, no padding (at most 2-way).
__host__ __device__ constexpr int right_key_words(int w) { return w + ((w + 15) >> 4) * 4; }
__host__ __device__ constexpr int right_key_pad(int seg, int form) {
    return form != kFormBytes16 ? 0 : seg >= 16 ? 2 : seg == 8 ? 4 : 0;
}
__device__ __forceinline__ int right_key_index(int a, int pad) { return a + (a >> 4) * pad; }

// The disparity loop of one image row: every pixel's first-minimum key, its
// neighbours' sums and (LR) the row's right-view keys into shared memory. The
// path count and slab form are template parameters, so each variant is its own
// straight-line loop with no per-round dispatch.
template <int NP, int FORM>
__device__ __forceinline__ void wta_row(const PairDev& pr, int y, uint32_t* right_key, int pad, uint32_t* best_key,
                                        uint32_t* nbr, uint16_t* sums) {
    constexpr int K = wta_disparities_per_lane(FORM);   // disparities a lane sums per round
    constexpr bool WIDE = FORM == kFormWide;
    const int W = pr.width, D = pr.nd;
    const bool lr = pr.lr_check != 0;
    const int chunks = pr.nd_vec / K;               // K-disparity chunks per pixel
    const int seg = wta_lanes_per_pixel(pr.nd_vec, FORM);
    const int rounds = (chunks + seg - 1) / seg;    // chunks per lane (wide D = 256: 8 lanes x 4; bytes: 1)
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwarps = blockDim.x >> 5;
    const int sub = lane / seg, c = lane % seg;
    const int ppw = 32 / seg;
    const RowView rv{pr.slabs, pr.shadow, pr.slab_stride, pr.shadow_stride, pr.nd_pad, pr.nd_vec, pr.shadow_cap};

    // This warp's sums of the current pixels: ppw rows of K * seg * rounds u16
    // (S(d) at d), read back for S(bd-1) and S(bd+1).
    uint16_t* const srow_p = sums + warp * kWtaSumsPerWarp + sub * (K * seg * rounds);
    for (int xb = warp * ppw; xb < W; xb += nwarps * ppw) {
        const int x = xb + sub;
        const bool actx = x < W;
        const size_t pix = (size_t)y * W + (actx ? x : 0);
        uint32_t best = 0xFFFFFFFFu;
        unsigned em = 0u;                           // escaped paths of the pixel (from round 0)
        for (int r = 0; r < rounds; ++r) {
            const int cc = r * seg + c;             // this lane's chunk: d = K cc .. K cc + K-1
            const bool act = actx && cc < chunks;
            uint32_t acc[K / 2];                    // acc[k] = S(K cc + 2k) | S(K cc + 2k+1) << 16
            if constexpr (K == 8) {
                acc[0] = acc[1] = acc[2] = acc[3] = 0u;
                if (r == 0) sum_paths<NP, WIDE, true>(rv, pix, cc, act, sub * seg, em, acc);
                else        sum_paths<NP, WIDE, false>(rv, pix, cc, act, sub * seg, em, acc);
            } else {
                if (r == 0) sum_bytes16<NP, true>(rv, pix, cc, act, sub * seg, em, acc);
                else        sum_bytes16<NP, false>(rv, pix, cc, act, sub * seg, em, acc);
            }
#pragma unroll
            for (int q = 0; q < K / 8; ++q)
                *reinterpret_cast<uint4*>(srow_p + K * cc + 8 * q) =
                    make_uint4(acc[4 * q], acc[4 * q + 1], acc[4 * q + 2], acc[4 * q + 3]);
            // key = S(d) << 8 | d (one byte permute: d in byte 0, S in bytes 1-2;
            // d = K cc + j < 256), whose minimum is the first minimum.
            const uint32_t d0 = (uint32_t)(K * cc);
            uint32_t key[K];
#pragma unroll
            for (int k = 0; k < K / 2; ++k) {
                key[2 * k] = __byte_perm(acc[k], d0 + 2 * k, 0x5104);
                key[2 * k + 1] = __byte_perm(acc[k], d0 + 2 * k + 1, 0x5324);
            }
            const int nb = (act ? D : 0) - (int)d0; // this lane's keys j < nb take part
            if (nb >= K) {                          // no pads: three-way minima
#pragma unroll
                for (int j = 0; j + 1 < K; j += 2) best = __vimin3_u32(best, key[j], key[j + 1]);
            } else {
#pragma unroll
                for (int j = 0; j < K; ++j)
                    if (j < nb) best = min(best, key[j]);
            }
            if (lr && act) {
                const int xr = x - K * cc;          // right-view column of this lane's d = K cc
                const int nr = min(D - K * cc, xr + 1);   // j < nr: d < D and x - d >= 0
                if (nr >= K) {
#pragma unroll
                    for (int j = 0; j < K; ++j) atomicMin(&right_key[right_key_index(xr - j, pad)], key[j]);
                } else {
#pragma unroll
                    for (int j = 0; j < K; ++j)
                        if (j < nr) atomicMin(&right_key[right_key_index(xr - j, pad)], key[j]);
                }
            }
        }
        for (int o = seg >> 1; o > 0; o >>= 1) best = min(best, __shfl_xor_sync(kFull, best, o));
        __syncwarp();                               // the pixel's sums are in shared memory
        if (c == 0 && actx) {
            // S(bd-1) and S(bd+1) (only used when 0 < bd < D-1, so both exist).
            const int bd = (int)(best & 0xFFu);
            const uint32_t c0 = srow_p[max(bd - 1, 0)], c2 = srow_p[min(bd + 1, D - 1)];
            best_key[x] = best;
            nbr[x] = c0 | (c2 << 16);
        }
        __syncwarp();                               // before the next pixels' sums
    }
}

// Four CTAs per SM (at most 64 registers a thread, no spills) keep enough slab loads in flight.
__global__ void __launch_bounds__(kWtaThreads, 4)
wta_kernel(const PairDev* __restrict__ pairs, int num_pairs) {
    extern __shared__ __align__(16) uint32_t smem[];
    const int k = find_wta_position(pairs, num_pairs, blockIdx.x);
    const int y = blockIdx.x - pairs[k].wta_row_begin;
    const PairDev pr = pairs[pairs[k].wta_pair];   // fields live in registers
    const int W = pr.width, D = pr.nd, P = pr.num_paths;
    const bool lr = pr.lr_check != 0;

    const int rk = right_key_words(W);
    uint32_t* right_key = smem;                               // rk words: padded right-view keys (LR only)
    uint32_t* best_key = smem + rk;                           // W: S(bd) << 8 | bd
    uint32_t* nbr = best_key + W;                             // W: S(bd-1) | S(bd+1) << 16
    // then the warps' sums (16-byte aligned)
    uint16_t* sums = reinterpret_cast<uint16_t*>(smem + ((rk + 2 * W + 3) & ~3));
    const int form = wta_form(pr.nd_vec, pr.wide_slabs != 0);   // the order groups pairs by (P, form)
    const int pad = right_key_pad(wta_lanes_per_pixel(pr.nd_vec, form), form);

    if (lr)
        for (int i = threadIdx.x; i < rk; i += blockDim.x) right_key[i] = 0xFFFFFFFFu;
    __syncthreads();

    const bool subpixel = pr.subpixel != 0;
    switch ((P == 2 ? 0 : P == 4 ? 1 : 2) * 3 + form) {   // uniform over the CTA
        case 0: wta_row<2, kFormBytes16>(pr, y, right_key, pad, best_key, nbr, sums); break;
        case 1: wta_row<2, kFormBytes8>(pr, y, right_key, pad, best_key, nbr, sums); break;
        case 2: wta_row<2, kFormWide>(pr, y, right_key, pad, best_key, nbr, sums); break;
        case 3: wta_row<4, kFormBytes16>(pr, y, right_key, pad, best_key, nbr, sums); break;
        case 4: wta_row<4, kFormBytes8>(pr, y, right_key, pad, best_key, nbr, sums); break;
        case 5: wta_row<4, kFormWide>(pr, y, right_key, pad, best_key, nbr, sums); break;
        case 6: wta_row<8, kFormBytes16>(pr, y, right_key, pad, best_key, nbr, sums); break;
        case 7: wta_row<8, kFormBytes8>(pr, y, right_key, pad, best_key, nbr, sums); break;
        default: wta_row<8, kFormWide>(pr, y, right_key, pad, best_key, nbr, sums); break;
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
        // The parabola step here, one pixel a thread, rather than in the lanes
        // c = 0 of the disparity loop.
        const uint32_t best = best_key[x];
        const int dl = (int)(best & 0xFFu);
        float v = (float)dl;
        if (subpixel && dl > 0 && dl < D - 1) {
            const uint32_t n = nbr[x];
            const float f0 = (float)(n & 0xFFFFu), f1 = (float)(best >> 8), f2 = (float)(n >> 16);
            const float denom = 2.0f * (f0 + f2 - 2.0f * f1);
            if (fabsf(denom) > 1e-6f) v = __fadd_rn(v, __fdiv_rn(f0 - f2, denom));
        }
        bool valid = true;
        if (lr) {
            const int xr = x - dl;
            valid = xr >= 0 && abs(dl - (int)(right_key[right_key_index(xr, pad)] & 0xFFu)) <= pr.lr_tolerance;
        }
        out[x] = valid ? v : pr.invalid_value;
        if (out_i) out_i[x] = (int16_t)(valid ? dl : -1);
        // Depth epilogue: depth = fx * baseline / disparity (the conversion the
        // reference leaves to its caller, kernels/sgm.rs:284-286).
        if (out_z)
            out_z[x] = (valid && v > 0.0f) ? __fdiv_rn(pr.depth_scale, v) : pr.depth_invalid;
    }
}

}  // namespace

size_t wta_smem_bytes(int max_width) {
    return ((size_t)right_key_words(max_width) + 2 * (size_t)max_width + 3) / 4 * 4 * sizeof(uint32_t) +
           (size_t)(kWtaThreads / 32) * kWtaSumsPerWarp * sizeof(uint16_t);
}

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
