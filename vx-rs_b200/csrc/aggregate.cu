// Path aggregation of semi-global matching, scanline-pair form: every path of
// every pair of a batch in ONE persistent launch over a work queue of (pair,
// path, 64-scanline) units. Large batches run this form (fewer instructions per
// path-pixel-disparity); plans with few units run the single-scanline form
// (aggregate_single.cu).
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
// Evaluation. With A_d = min(o0, o2, o3) (independent of the current pixel) and
// f_d = u16(Lp[d] + P1) = o1_{d+1}, one pixel is the chain
//     t_d = min(A_d, f_{d-1});  f_d = u16(t_d + C_d + P1 - m);  Lp[d] = u16(f_d - P1)
// whose critical path is one min and one add per disparity.
//
// Scanline pairs. Every thread carries TWO scanlines, their u16 values side by
// side in the halves of 32-bit words, and every step of the chain is one
// per-half instruction for both: min.u16x2, the three-way DPX minimum for A_d,
// and per-half wrapping adds (which are exactly the shader's ushort
// arithmetic). The state word of disparity d holds (Lp_lo[d], Lp_hi[d]).
// A scanline that starts at this pixel gets o3 = 0 and m = 0 for its half:
// then min(o0,o1,o2,o3) = 0 and Lp[d] = C whatever its state held before, so
// no state is ever cleared and idle halves need no masking.
//
// Mapping. The state of a thread (one 32-bit word per disparity) lives in
// tensor memory (TMEM): the thread's TMEM lane, one column per disparity, read
// and written 8 columns at a time by warp-collective tcgen05.ld/st. A warp
// takes 64 neighbouring scanlines of one (pair, path): lane i carries
// scanlines i (low half) and i + 32 (high half).
// Costs. The eight paths of a pair share C(x, y, d), so the cost kernel
// (cost.cu) writes it once per pair as a byte volume (Dv bytes a pixel, 64
// where x - d < 0, 0 in the pads); a thread reads its two scanlines' 8 costs of
// a group as one 8-byte load each, one group ahead, and packs them into the
// u16 halves with byte permutes. The border needs no second body.
//
// Output. Each group's results go to a byte tile in shared memory (one row of
// Dv bytes per scanline); after the pixel the warp writes the rows of its
// active scanlines to the path's byte slab with coalesced 8-byte stores. The
// values of a vector are bounded by the census cost plus P2 unless the
// in-place o1 term pulls them below m (then they wrap), so almost every vector
// fits bytes; one with a value of 255 or more gets 0xFF in byte 0 and its
// exact u16 values, read back from TMEM (the state after the pixel is the
// vector), go to the u16 shadow slab. Wide slabs get every vector that way.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <functional>

#include "kernels.cuh"
#include "launch.hpp"

namespace vxsgm {
namespace pairs {

namespace {

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ uint32_t vmin2(uint32_t a, uint32_t b) {
    uint32_t r;
    asm("min.u16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}

// Tensor-memory (TMEM) access for the per-scanline state. Warp w of the CTA owns
// TMEM lanes 32(w%4)..32(w%4)+31 (one lane per thread) and the columns of its
// warpgroup; disparity d is column d. tcgen05.ld is asynchronous: its registers
// are threaded through the wait so that no use can be scheduled before the data
// has arrived. The callers are warp-converged (uniform control flow).
struct Words8 {
    uint32_t w[8];
};
__device__ __forceinline__ Words8 tmem_ld8(uint32_t taddr) {
    Words8 r;
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r.w[0]), "=r"(r.w[1]), "=r"(r.w[2]), "=r"(r.w[3]), "=r"(r.w[4]), "=r"(r.w[5]),
                   "=r"(r.w[6]), "=r"(r.w[7])
                 : "r"(taddr));
    return r;
}
__device__ __forceinline__ void tmem_wait_ld(Words8& r) {
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r.w[0]), "+r"(r.w[1]), "+r"(r.w[2]), "+r"(r.w[3]), "+r"(r.w[4]), "+r"(r.w[5]),
                   "+r"(r.w[6]), "+r"(r.w[7])::"memory");
}
__device__ __forceinline__ void tmem_st8(uint32_t taddr, const Words8& v) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"r"(taddr),
                 "r"(v.w[0]), "r"(v.w[1]), "r"(v.w[2]), "r"(v.w[3]), "r"(v.w[4]), "r"(v.w[5]), "r"(v.w[6]),
                 "r"(v.w[7])
                 : "memory");
}
__device__ __forceinline__ void tmem_wait_st() {
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}

// Per-scanline constants of one unit (u16 values in both halves).
struct ScanConst {
    uint32_t p1x2;        // P1
    uint32_t np1x2;       // -P1 (mod 2^16)
    uint32_t p1p1x2;      // P1 + 1: P1 - m = (~m) + P1 + 1
    uint32_t p2x2;        // P2
    int Dp, G;            // disparities padded to 8, groups of 8
    int last_j;           // position of d = D-1 inside the last group (0..7)
};

// Per-pixel values shared by the groups of one pixel (both scanlines).
struct PixelState {
    uint32_t o3x2;   // u16(m + P2), 0 for a scanline that starts here
    uint32_t kc2;    // u16(P1 - m)
    uint32_t f;      // o1 of the next disparity
    uint32_t mn;     // running min of the new values (d < D)
    uint32_t mx;     // running max of the new values (d < D)
};

// One group of 8 disparities d = 8g..8g+7 of one pixel of both scanlines, in
// two parts so that the state of the next group (whose first word only the last
// disparity needs) can still be in flight during the first: head = d 8g..8g+6,
// tail = d 8g+7 and the group's minimum and maximum. S = old state words of the
// group, nxt = old state word of d = 8g+8 (unused for the last group), cw = the
// group's packed costs; out = the new words. LAST: the group holding d = D-1,
// whose o2 is forced to 0xFFFF and whose pads (d >= D) are kept out of the
// minimum and maximum.
// A_d = min(o0, o2, o3) and w_d = C_d + P1 - m of disparity j of the group:
// neither depends on the chain, so a whole group of them is formed first and
// the chain itself is two dependent instructions per disparity.
template <bool LAST>
__device__ __forceinline__ void group_pre(const uint32_t s, const uint32_t sn, const uint32_t c, const int j,
                                          const ScanConst& k, const PixelState& ps, uint32_t& A, uint32_t& w) {
    uint32_t o2 = __vadd2(sn, k.p1x2);
    if (LAST && j == k.last_j) o2 = 0xFFFFFFFFu;
    A = __vimin3_u16x2(s, o2, ps.o3x2);
    w = __vadd2(c, ps.kc2);
}
// The chain: t = min(A_d, f_{d-1}), f_d = t + w_d, Lp[d] = f_d - P1.
__device__ __forceinline__ void chain_step(const uint32_t A, const uint32_t w, const ScanConst& k,
                                           PixelState& ps, uint32_t& o) {
    ps.f = __vadd2(vmin2(A, ps.f), w);
    o = __vadd2(ps.f, k.np1x2);
}
template <bool LAST>
__device__ __forceinline__ void sgm_group_head(const Words8& S, const uint32_t (&cw)[8], const ScanConst& k,
                                               PixelState& ps, Words8& out, uint32_t& w7) {
    uint32_t A[7], w[7];
#pragma unroll
    for (int j = 0; j < 7; ++j) group_pre<LAST>(S.w[j], S.w[j + 1], cw[j], j, k, ps, A[j], w[j]);
    w7 = __vadd2(cw[7], ps.kc2);
#pragma unroll
    for (int j = 0; j < 7; ++j) chain_step(A[j], w[j], k, ps, out.w[j]);
}
template <bool LAST>
__device__ __forceinline__ void sgm_group_tail(const Words8& S, const uint32_t nxt, const uint32_t w7,
                                               const ScanConst& k, PixelState& ps, Words8& out) {
    uint32_t o2 = __vadd2(nxt, k.p1x2);
    if (LAST && k.last_j == 7) o2 = 0xFFFFFFFFu;
    chain_step(__vimin3_u16x2(S.w[7], o2, ps.o3x2), w7, k, ps, out.w[7]);
    if (!LAST) {
#pragma unroll
        for (int j = 0; j < 8; j += 2) {
            ps.mn = __vimin3_u16x2(ps.mn, out.w[j], out.w[j + 1]);
            ps.mx = __vimax3_u16x2(ps.mx, out.w[j], out.w[j + 1]);
        }
    } else {
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            if (j <= k.last_j) {                   // pads never count
                ps.mn = vmin2(ps.mn, out.w[j]);
                ps.mx = __vmaxu2(ps.mx, out.w[j]);
            }
        }
    }
}

// Byte rows of one group: the low bytes of the 8 words' low halves (scanline
// lo) and of their high halves (scanline hi), d-ascending.
__device__ __forceinline__ void group_bytes(const Words8& o, uint2& lo, uint2& hi) {
    const uint32_t t01 = __byte_perm(o.w[0], o.w[1], 0x6420);   // lo0 hi0 lo1 hi1
    const uint32_t t23 = __byte_perm(o.w[2], o.w[3], 0x6420);
    const uint32_t t45 = __byte_perm(o.w[4], o.w[5], 0x6420);
    const uint32_t t67 = __byte_perm(o.w[6], o.w[7], 0x6420);
    lo.x = __byte_perm(t01, t23, 0x6420);
    hi.x = __byte_perm(t01, t23, 0x7531);
    lo.y = __byte_perm(t45, t67, 0x6420);
    hi.y = __byte_perm(t45, t67, 0x7531);
}

// Packed costs of disparities 4i..4i+3 (one word of each scanline's cost row):
// cw = C_lo | C_hi << 16 by one byte permute each; the costs are at most 64, so
// the sign-replicating selector bytes give the zero high bytes.
__device__ __forceinline__ uint32_t prmt(uint32_t a, uint32_t b, uint32_t sel) {
    uint32_t r;
    asm("prmt.b32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(sel));
    return r;
}
__device__ __forceinline__ void cost_words(uint32_t (&cw)[8], const uint2 lo, const uint2 hi) {
    cw[0] = prmt(lo.x, hi.x, 0xC480u);
    cw[1] = prmt(lo.x, hi.x, 0xD591u);
    cw[2] = prmt(lo.x, hi.x, 0xE6A2u);
    cw[3] = prmt(lo.x, hi.x, 0xF7B3u);
    cw[4] = prmt(lo.y, hi.y, 0xC480u);
    cw[5] = prmt(lo.y, hi.y, 0xD591u);
    cw[6] = prmt(lo.y, hi.y, 0xE6A2u);
    cw[7] = prmt(lo.y, hi.y, 0xF7B3u);
}

// One pixel of the 64 scanlines of a warp (all lanes execute it: the TMEM
// accesses are warp-collective). tstate = this warp's TMEM address (lane field
// = its first lane, column 0). cv_lo / cv_hi = the two scanlines' rows of the
// pair's cost volume at this pixel (Dv bytes each, 64 already in place where
// x - d < 0). m = the previous pixel's minimum per half; start = 0xFFFF in each
// half whose scanline starts at this pixel. row_lo / row_hi = the two
// scanlines' rows of the warp's output tile (u16 values when WIDE, else bytes).
// Returns the per-half maximum of the new vector (d < D). Software pipeline over
// groups (loop unrolled by two, register sets in ping-pong): the costs come in
// 16-byte loads of two groups a scanline (each lane reads its own rows, so one
// load instruction touches 32 cache lines: halving the load count halves that
// traffic), the pair after the current one in flight while it runs; the state
// of group g+1 is in flight while group g runs its chain (waited for only
// before g's last disparity), and g+1's packed costs are formed right after
// g's chain. Reading 16 bytes never leaves the Dv-byte row (Dv = D rounded up
// to 16).
template <bool WIDE>
__device__ __forceinline__ uint32_t sgm_pixel(const uint32_t tstate, uint32_t& m, const uint32_t start,
                                                 const uint8_t* __restrict__ cv_lo,
                                                 const uint8_t* __restrict__ cv_hi,
                                                 const uint8_t* __restrict__ nx_lo,
                                                 const uint8_t* __restrict__ nx_hi, uint4& g0_lo, uint4& g0_hi,
                                                 const ScanConst& k, unsigned char* __restrict__ row_lo,
                                                 unsigned char* __restrict__ row_hi) {
    PixelState ps;
    const uint32_t m0 = m & ~start;
    ps.o3x2 = __vadd2(m0, k.p2x2) & ~start;
    ps.kc2 = __vadd2(~m0, k.p1p1x2);
    ps.f = 0xFFFFFFFFu;            // o1 at d = 0
    ps.mn = 0xFFFFFFFFu;
    ps.mx = 0u;
    auto load = [&](uint4& lo, uint4& hi, int g) {   // groups g, g+1 (g even)
        lo = __ldg(reinterpret_cast<const uint4*>(cv_lo + 8 * g));
        hi = __ldg(reinterpret_cast<const uint4*>(cv_hi + 8 * g));
    };
    auto store = [&](const Words8& o, int g) {
        if (WIDE) {             // u16 rows: 8 values (16 bytes) per group
            *reinterpret_cast<uint4*>(row_lo + 16 * g) = make_uint4(
                __byte_perm(o.w[0], o.w[1], 0x5410), __byte_perm(o.w[2], o.w[3], 0x5410),
                __byte_perm(o.w[4], o.w[5], 0x5410), __byte_perm(o.w[6], o.w[7], 0x5410));
            *reinterpret_cast<uint4*>(row_hi + 16 * g) = make_uint4(
                __byte_perm(o.w[0], o.w[1], 0x7632), __byte_perm(o.w[2], o.w[3], 0x7632),
                __byte_perm(o.w[4], o.w[5], 0x7632), __byte_perm(o.w[6], o.w[7], 0x7632));
        } else {                // byte rows: 8 bytes per group
            uint2 lo, hi;
            group_bytes(o, lo, hi);
            *reinterpret_cast<uint2*>(row_lo + 8 * g) = lo;
            *reinterpret_cast<uint2*>(row_hi + 8 * g) = hi;
        }
        tmem_st8(tstate + 8 * g, o);
    };
    uint4 q_l = g0_lo, q_h = g0_hi, n_l, n_h;      // groups 0 and 1, loaded during the previous pixel
    uint32_t ca[8], cb[8];
    Words8 oa, ob;
    uint32_t w7;
    Words8 sa = tmem_ld8(tstate), sb;
    cost_words(ca, make_uint2(q_l.x, q_l.y), make_uint2(q_h.x, q_h.y));
    tmem_wait_ld(sa);
    int g = 0;
#pragma unroll 1
    for (; g + 2 < k.G; g += 2) {
        load(n_l, n_h, g + 2);                       // groups g+2, g+3 in flight
        sb = tmem_ld8(tstate + 8 * (g + 1));
        sgm_group_head<false>(sa, ca, k, ps, oa, w7);
        tmem_wait_ld(sb);
        sgm_group_tail<false>(sa, sb.w[0], w7, k, ps, oa);
        store(oa, g);
        cost_words(cb, make_uint2(q_l.z, q_l.w), make_uint2(q_h.z, q_h.w));
        sa = tmem_ld8(tstate + 8 * (g + 2));
        sgm_group_head<false>(sb, cb, k, ps, ob, w7);
        tmem_wait_ld(sa);
        sgm_group_tail<false>(sb, sa.w[0], w7, k, ps, ob);
        store(ob, g + 1);
        q_l = n_l;
        q_h = n_h;
        cost_words(ca, make_uint2(q_l.x, q_l.y), make_uint2(q_h.x, q_h.y));
    }
    // The next pixel's groups 0 and 1 (nx_lo / nx_hi: its rows, or any valid row).
    g0_lo = __ldg(reinterpret_cast<const uint4*>(nx_lo));
    g0_hi = __ldg(reinterpret_cast<const uint4*>(nx_hi));
    if (g + 1 < k.G) {
        sb = tmem_ld8(tstate + 8 * (g + 1));
        sgm_group_head<false>(sa, ca, k, ps, oa, w7);
        tmem_wait_ld(sb);
        sgm_group_tail<false>(sa, sb.w[0], w7, k, ps, oa);
        store(oa, g);
        cost_words(cb, make_uint2(q_l.z, q_l.w), make_uint2(q_h.z, q_h.w));
        sgm_group_head<true>(sb, cb, k, ps, ob, w7);
        sgm_group_tail<true>(sb, 0u, w7, k, ps, ob);
        store(ob, g + 1);
    } else {
        sgm_group_head<true>(sa, ca, k, ps, oa, w7);
        sgm_group_tail<true>(sa, 0u, w7, k, ps, oa);
        store(oa, g);
    }
    tmem_wait_st();            // the next pixel reads this state back
    m = ps.mn;
    return ps.mx;
}

__device__ __forceinline__ ScanConst scan_const(const PairDev& pr) {
    ScanConst k;
    const uint32_t P1 = (uint32_t)pr.p1, P2 = (uint32_t)pr.p2;
    k.p1x2 = P1 | (P1 << 16);
    const uint32_t np1 = (0x10000u - P1) & 0xFFFFu;
    k.np1x2 = np1 | (np1 << 16);
    const uint32_t p1p1 = (P1 + 1u) & 0xFFFFu;
    k.p1p1x2 = p1p1 | (p1p1 << 16);
    k.p2x2 = P2 | (P2 << 16);
    k.Dp = pr.nd_pad;
    k.G = pr.nd_pad / 8;
    k.last_j = (pr.nd - 1) - 8 * (k.G - 1);
    return k;
}

// Writes the rows la..lb (a run of active scanlines, 0..63) of the warp's
// tile to the slab: row r's vector (vb bytes) goes to dst0 + r * stride. The
// rows' 8-byte chunks are distributed over the lanes in address order (chunk
// c = (r - la) * V + h, walked with a running (r, h): no division per chunk),
// so consecutive lanes write consecutive 8 bytes of a vector. Streaming stores:
// the slabs are read once by the WTA kernel and must not push the cost volume,
// which every path of the pair re-reads, out of L2.
__device__ __forceinline__ void flush_tile(const unsigned char* __restrict__ tile, int row_bytes, int vb,
                                           int la, int lb, unsigned char* __restrict__ dst0, size_t stride,
                                           int lane) {
    const int V = vb / 8;
    const int n = (lb - la + 1) * V;
    const int q = 32 / V, rr = 32 % V;
    int r = la + lane / V, h = lane % V;
    for (int c = lane; c < n; c += 32) {
        __stcs(reinterpret_cast<uint2*>(dst0 + (size_t)r * stride + 8 * h),
               *reinterpret_cast<const uint2*>(tile + r * row_bytes + 8 * h));
        h += rr;
        r += q;
        if (h >= V) {
            h -= V;
            ++r;
        }
    }
}

// The lanes whose w_lo / w_hi is set write their scanlines' exact u16 vectors,
// read back from TMEM (the state after the pixel), to sh_lo / sh_hi (in the
// shadow or wide slab). All lanes take part in the TMEM loads.
__device__ __forceinline__ void write_u16_vectors(uint32_t tstate, int G, bool w_lo, bool w_hi,
                                                  uint16_t* __restrict__ sh_lo, uint16_t* __restrict__ sh_hi) {
    for (int g = 0; g < G; ++g) {
        Words8 s = tmem_ld8(tstate + 8 * g);
        tmem_wait_ld(s);
        if (w_lo) {
            const uint4 v = make_uint4(__byte_perm(s.w[0], s.w[1], 0x5410), __byte_perm(s.w[2], s.w[3], 0x5410),
                                       __byte_perm(s.w[4], s.w[5], 0x5410), __byte_perm(s.w[6], s.w[7], 0x5410));
            __stcs(reinterpret_cast<uint4*>(sh_lo + 8 * g), v);
        }
        if (w_hi) {
            const uint4 v = make_uint4(__byte_perm(s.w[0], s.w[1], 0x7632), __byte_perm(s.w[2], s.w[3], 0x7632),
                                       __byte_perm(s.w[4], s.w[5], 0x7632), __byte_perm(s.w[6], s.w[7], 0x7632));
            __stcs(reinterpret_cast<uint4*>(sh_hi + 8 * g), v);
        }
    }
}

// After one pixel step: the rows of the active run go to the path's slab.
// Byte slabs: a vector with a value of 255 or more (escape) gets the marker in
// byte 0 of its row and its shadow slot in bytes 4..7, and its exact u16
// values are read back from TMEM to that slot (nothing is written when the
// pair's shadow pool has run out). Wide slabs: the tile rows are the u16 vectors. pix0 = pixel of
// tile row 0; pix_lo / pix_hi = this lane's two scanlines' pixels (used only for
// an active scanline); pstride = pixel stride between tile rows (1 or W).
// CP (compact): the batch has pairs whose escaped vectors go to a shadow pool;
// their rows carry the slot, which the WTA kernel reads. Without CP every
// escaped vector goes to its pixel's place in the full shadow (the slot the
// WTA kernel computes for a pair without a pool), and the pixel loop has none
// of the pool's bookkeeping.
template <bool CP>
__device__ __forceinline__ void finish_pixel(const PairDev& pr, const EscapeTarget& et, int path, bool wide, int Dv,
                                             uint32_t tstate, int G, uint32_t mx, bool act_lo, bool act_hi,
                                             const unsigned char* tile, int row_bytes, unsigned char* row_lo,
                                             unsigned char* row_hi, size_t pix0, size_t pstride, size_t pix_lo,
                                             size_t pix_hi, int lane) {
    const bool esc_lo = !wide && act_lo && (mx & 0xFFFFu) >= 0xFFu;
    const bool esc_hi = !wide && act_hi && (mx >> 16) >= 0xFFu;
    uint32_t slot_lo = kNoSlot, slot_hi = kNoSlot;
    if constexpr (CP) {
        if (esc_lo) {
            slot_lo = take_slot(et, pix_lo);
            row_lo[0] = 0xFFu;
            *reinterpret_cast<uint32_t*>(row_lo + 4) = slot_lo;  // rows are 8-byte aligned
        }
        if (esc_hi) {
            slot_hi = take_slot(et, pix_hi);
            row_hi[0] = 0xFFu;
            *reinterpret_cast<uint32_t*>(row_hi + 4) = slot_hi;
        }
    } else {
        if (esc_lo) row_lo[0] = 0xFFu;
        if (esc_hi) row_hi[0] = 0xFFu;
    }
    const unsigned al = __ballot_sync(kFull, act_lo), ah = __ballot_sync(kFull, act_hi);
    const unsigned e = __ballot_sync(kFull, esc_lo || esc_hi);
    __syncwarp();
    if (al | ah) {
        // The active scanlines are one run of rows: the low and high runs join.
        const unsigned long long act = (unsigned long long)al | ((unsigned long long)ah << 32);
        const int la = __ffsll((long long)act) - 1, lb = 63 - __clzll((long long)act);
        if (wide) {
            const int Dp = pr.nd_pad;
            unsigned char* dst = reinterpret_cast<unsigned char*>(pr.shadow + pr.shadow_stride * (size_t)path +
                                                                  pix0 * Dp);
            flush_tile(tile, row_bytes, 2 * Dp, la, lb, dst, pstride * Dp * 2, lane);
        } else {
            unsigned char* dst = pr.slabs + pr.slab_stride * (size_t)path + pix0 * Dv;
            flush_tile(tile, row_bytes, Dv, la, lb, dst, pstride * Dv, lane);
        }
    }
    if (e) {
        if constexpr (CP) {
            const bool w_lo = esc_lo && slot_lo != kNoSlot, w_hi = esc_hi && slot_hi != kNoSlot;
            write_u16_vectors(tstate, G, w_lo, w_hi, et.shadow + (w_lo ? (size_t)slot_lo * et.Dp : 0),
                              et.shadow + (w_hi ? (size_t)slot_hi * et.Dp : 0));
        } else {
            uint16_t* base = pr.shadow + pr.shadow_stride * (size_t)path;
            write_u16_vectors(tstate, G, esc_lo, esc_hi, base + pix_lo * pr.nd_pad, base + pix_hi * pr.nd_pad);
        }
    }
    __syncwarp();
}

// Unit = 64 scanlines of a vertical or diagonal path. WT: the batch has
// wide-slab pairs (the u16 body is compiled in).
template <bool WT, bool CP>
__device__ __forceinline__ void run_vertical_unit(const PairDev& pr, const JobDev& job, int first,
                                                  uint32_t tstate, unsigned char* __restrict__ tile,
                                                  int row_bytes) {
    const int lane = threadIdx.x & 31;
    const int W = pr.width, H = pr.height;
    const ScanConst k = scan_const(pr);
    const int Dv = pr.nd_vec;
    const bool wide = WT && pr.wide_slabs != 0;
    const int dx = job.dx, dy = job.dy;
    const EscapeTarget et = CP ? escape_target(pr, job.path) : EscapeTarget{};

    const int k0 = job.k_min + first;         // scanline index of tile row 0
    // This lane's two scanlines (tile rows lane and lane + 32): a scanline's
    // pixel at step t is x = kk + dx*t, y = y0 + dy*t (vertical: dx = 0).
    const int y0 = dy > 0 ? 0 : H - 1;
    auto range = [&](int i, int& tb, int& te) {
        const int kk = k0 + i;
        if (first + i >= job.num_scanlines) { tb = 0x7fffffff; te = -1; return; }
        if (dx == 0) { tb = 0; te = H; }
        else if (dx > 0) { tb = max(0, -kk); te = min(H, W - kk); }
        else { tb = max(0, kk - W + 1); te = min(H, kk + 1); }
    };
    int tb_lo, te_lo, tb_hi, te_hi;
    range(lane, tb_lo, te_lo);
    range(lane + 32, tb_hi, te_hi);
    const int t_lo = __reduce_min_sync(kFull, min(tb_lo, tb_hi));
    const int t_hi = __reduce_max_sync(kFull, max(te_lo, te_hi));
    if (t_lo >= t_hi) return;

    const uint8_t* __restrict__ CV = pr.costs;
    uint32_t m = 0u;
    // Costs from the pair's cost volume: the two scanlines' rows at the step's
    // pixels (a half outside its scanline reads pixel 0's row, in bounds and
    // unused: it restarts from L = C where its scanline begins).
    unsigned char* row_lo = tile + lane * row_bytes;
    unsigned char* row_hi = tile + (lane + 32) * row_bytes;
    // Cost rows of step t's two scanlines (pixel 0's row for a half outside its scanline).
    auto rows_at = [&](int t, const uint8_t*& lo, const uint8_t*& hi) {
        const size_t p0 = (size_t)((ptrdiff_t)(y0 + dy * t) * W + k0 + dx * t);
        lo = CV + (t >= tb_lo && t < te_lo ? (p0 + lane) * Dv : 0);
        hi = CV + (t >= tb_hi && t < te_hi ? (p0 + lane + 32) * Dv : 0);
    };
    const uint8_t *cv_lo, *cv_hi;
    rows_at(t_lo, cv_lo, cv_hi);
    uint4 g0_lo = __ldg(reinterpret_cast<const uint4*>(cv_lo)), g0_hi = __ldg(reinterpret_cast<const uint4*>(cv_hi));
    for (int t = t_lo; t < t_hi; ++t) {
        const bool act_lo = t >= tb_lo && t < te_lo, act_hi = t >= tb_hi && t < te_hi;
        const uint32_t start = (t == tb_lo ? 0x0000FFFFu : 0u) | (t == tb_hi ? 0xFFFF0000u : 0u);
        const int xb = k0 + dx * t;             // x of tile row 0
        const int y = y0 + dy * t;
        const size_t pix0 = (size_t)((ptrdiff_t)y * W + xb);
        const uint8_t *nx_lo = CV, *nx_hi = CV;
        if (t + 1 < t_hi) rows_at(t + 1, nx_lo, nx_hi);
        const uint32_t mx =
            wide ? sgm_pixel<true>(tstate, m, start, cv_lo, cv_hi, nx_lo, nx_hi, g0_lo, g0_hi, k, row_lo, row_hi)
                 : sgm_pixel<false>(tstate, m, start, cv_lo, cv_hi, nx_lo, nx_hi, g0_lo, g0_hi, k, row_lo, row_hi);
        cv_lo = nx_lo;
        cv_hi = nx_hi;
        finish_pixel<CP>(pr, et, job.path, wide, Dv, tstate, k.G, mx, act_lo, act_hi, tile, row_bytes, row_lo,
                         row_hi, pix0, 1, pix0 + lane, pix0 + lane + 32, lane);
    }
}

// Unit = 64 rows of a horizontal path.
template <bool WT, bool CP>
__device__ __forceinline__ void run_horizontal_unit(const PairDev& pr, const JobDev& job, int first,
                                                    uint32_t tstate, unsigned char* __restrict__ tile,
                                                    int row_bytes) {
    const int lane = threadIdx.x & 31;
    const int W = pr.width;
    const ScanConst k = scan_const(pr);
    const int Dv = pr.nd_vec;
    const bool wide = WT && pr.wide_slabs != 0;
    const int dx = job.dx;
    const EscapeTarget et = CP ? escape_target(pr, job.path) : EscapeTarget{};
    const bool act_lo = first + lane < job.num_scanlines;
    const bool act_hi = first + 32 + lane < job.num_scanlines;
    const uint8_t* __restrict__ CV = pr.costs;
    uint32_t m = 0u;
    const int x0 = dx > 0 ? 0 : W - 1;
    // Costs from the pair's cost volume: rows first + lane and first + 32 + lane
    // at column x (a row past the image reads pixel 0's row, unused).
    unsigned char* row_lo = tile + lane * row_bytes;
    unsigned char* row_hi = tile + (lane + 32) * row_bytes;
    // Column x's cost rows of the two scanlines (pixel 0's row for a row past the image).
    const uint8_t* cv_lo = CV + (act_lo ? ((size_t)(first + lane) * W + x0) * Dv : 0);
    const uint8_t* cv_hi = CV + (act_hi ? ((size_t)(first + 32 + lane) * W + x0) * Dv : 0);
    const ptrdiff_t step_lo = act_lo ? (ptrdiff_t)dx * Dv : 0, step_hi = act_hi ? (ptrdiff_t)dx * Dv : 0;
    uint4 g0_lo = __ldg(reinterpret_cast<const uint4*>(cv_lo)), g0_hi = __ldg(reinterpret_cast<const uint4*>(cv_hi));
    for (int t = 0; t < W; ++t) {
        const int x = x0 + dx * t;
        const uint32_t start = t == 0 ? 0xFFFFFFFFu : 0u;
        const size_t pix0 = (size_t)first * W + x;
        const bool more = t + 1 < W;
        const uint8_t* nx_lo = more ? cv_lo + step_lo : CV;
        const uint8_t* nx_hi = more ? cv_hi + step_hi : CV;
        const uint32_t mx =
            wide ? sgm_pixel<true>(tstate, m, start, cv_lo, cv_hi, nx_lo, nx_hi, g0_lo, g0_hi, k, row_lo, row_hi)
                 : sgm_pixel<false>(tstate, m, start, cv_lo, cv_hi, nx_lo, nx_hi, g0_lo, g0_hi, k, row_lo, row_hi);
        cv_lo = nx_lo;
        cv_hi = nx_hi;
        // Rows first..first+63, one vector per row at column x.
        finish_pixel<CP>(pr, et, job.path, wide, Dv, tstate, k.G, mx, act_lo, act_hi, tile, row_bytes, row_lo,
                         row_hi, pix0, (size_t)W, pix0 + (size_t)lane * W, pix0 + (size_t)(lane + 32) * W, lane);
    }
}

}  // namespace

// Unit range of queue class c (c < kMaxQueueClasses), read with constant
// indices so that the parameter struct stays in the constant bank.
__device__ __forceinline__ void class_range(const AggQueues& q, int c, int& b, int& e) {
    b = c == 0 ? q.begin[0] : c == 1 ? q.begin[1] : c == 2 ? q.begin[2] : q.begin[3];
    e = c == 0 ? q.begin[1] : c == 1 ? q.begin[2] : c == 2 ? q.begin[3] : q.begin[4];
}

template <bool WT, bool CP>
__global__ void __launch_bounds__(kAggMaxThreads)
aggregate_kernel(const PairDev* __restrict__ pairs, const JobDev* __restrict__ jobs,
                 const UnitDev* __restrict__ units, const AggQueues q, unsigned* __restrict__ counters,
                 int dp_max, int tmem_cols) {
    extern __shared__ __align__(16) unsigned char agg_smem[];
    __shared__ uint32_t tmem_base;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int row_bytes = aggregate_row_bytes(dp_max, WT);
    // The warps' tiles start aggregate_tile_offset(dp_max) bytes in (unused):
    // compiled with that batch-dependent base, the pixel loop measured 3 %
    // faster (18.2 vs 18.8 ms on the 64-pair mixed batch) than with base 0.
    unsigned char* tile = agg_smem + aggregate_tile_offset(dp_max) + (size_t)warp * aggregate_warp_smem(dp_max, WT);

    // TMEM for the state of all the CTA's scanlines, allocated by warp 0 for the
    // whole persistent loop and released by warp 0 after every warp is done.
    // Warp w owns TMEM lanes 32*(w%4).. (its lane quarter) and, inside them, the
    // columns of its warpgroup w/4, from q.col0[w/4] on (its class budget).
    if (warp == 0) {
        const unsigned slot = (unsigned)__cvta_generic_to_shared(&tmem_base);
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot),
                     "r"(tmem_cols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const int wg = warp >> 2;
    const int col0 = wg == 0 ? q.col0[0] : wg == 1 ? q.col0[1] : wg == 2 ? q.col0[2] : q.col0[3];
    const uint32_t tstate = tmem_base + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)col0;

    int c = wg == 0 ? q.first_class[0] : wg == 1 ? q.first_class[1] : wg == 2 ? q.first_class[2] : q.first_class[3];
    int cb, ce;
    class_range(q, c, cb, ce);
    for (;;) {
        int u = 0;
        if (lane == 0) u = (int)atomicAdd(&counters[c], 1u);
        u = __shfl_sync(kFull, u, 0);
        if (u >= ce - cb) {          // this class is empty: the next smaller one
            if (++c >= q.n_classes) break;
            class_range(q, c, cb, ce);
            continue;
        }
        const UnitDev unit = units[cb + u];
        const JobDev job = jobs[unit.job];
        const PairDev& pr = pairs[job.pair];
        if (job.dy == 0)
            run_horizontal_unit<WT, CP>(pr, job, unit.first_scanline, tstate, tile, row_bytes);
        else
            run_vertical_unit<WT, CP>(pr, job, unit.first_scanline, tstate, tile, row_bytes);
        __syncwarp();
    }

    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base),
                     "r"(tmem_cols));
    }
}

// The kernel for a batch's tile format and shadow kind (the census word width
// does not matter: the costs come from the volume).
const void* aggregate_kernel_fn(bool wide_tiles, bool compact) {
    if (compact) return wide_tiles ? (const void*)aggregate_kernel<true, true> : (const void*)aggregate_kernel<false, true>;
    return wide_tiles ? (const void*)aggregate_kernel<true, false> : (const void*)aggregate_kernel<false, false>;
}

// Launch shape of the aggregation kernel: one CTA per SM (the CUDA occupancy
// calculator allows one CTA per SM for a kernel that allocates tensor memory)
// with as many warpgroups as the SM's 512 TMEM columns, registers and shared
// memory hold. A warpgroup's 4 warps cover the 128 TMEM lanes (256 scanlines)
// and need one column per padded disparity of the units they run: its column
// budget. Budgets are per warpgroup, so a batch mixing D = 192 with smaller D
// can run three warpgroups (192 + 192 + 128 columns) where uniform budgets of
// the largest D would allow two.

// Largest number of warpgroups one aggregation CTA can hold for a batch whose
// padded D lie in [dp_min, dp_max]: one budget of dp_max and the rest of the
// 512 TMEM columns in budgets of dp_min, the registers, and the shared memory
// of an SM (every warp's output tile is sized for dp_max).
int max_warpgroups(int dp_max, int dp_min, bool wide_tiles) {
    const int by_tmem = 1 + (512 - dp_max) / std::max(dp_min, 8);
    int regs = 128, regs_sm = 65536, dev = 0, smem_sm = 227 * 1024;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev);
    cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    // Either shadow kind may run with the shape chosen here: the larger register count counts.
    for (bool compact : {false, true}) {
        cudaFuncAttributes fa{};
        if (cudaFuncGetAttributes(&fa, aggregate_kernel_fn(wide_tiles, compact)) == cudaSuccess &&
            fa.numRegs > 0)
            regs = compact ? std::max(regs, fa.numRegs) : fa.numRegs;
    }
    cudaGetLastError();
    const int by_regs = regs_sm / (regs * 128);
    const int by_smem =
        (int)((smem_sm - 1024 - (int)aggregate_tile_offset(dp_max)) / (4 * aggregate_warp_smem(dp_max, wide_tiles)));
    return std::max(1, std::min({by_tmem, by_regs, by_smem, kAggMaxWarpgroups}));
}

// Column budgets of `warpgroups` warpgroups for a batch whose units need the
// padded disparity counts dps[0] > dps[1] > ... (n_dps distinct values) with
// work[i] the share of the queued work (sum of longest scanline x D over the
// units) of the units needing dps[i]. Budgets are non-increasing, each one of
// dps (the first dps[0]), and sum to at most 512 columns. The units needing
// dps[j] or more can only run on warpgroups whose budget is at least dps[j]:
// with n_j such warpgroups out of W and a share F_j of the work, they need
// F_j * W / n_j of the time a perfectly shared queue would take. The budgets
// minimise the largest such ratio (ties: larger budgets, more flexible); the
// ratio (>= 1) is returned, and the budgets in cols[0..warpgroups-1]. Returns
// 0 when no budgets of that many warpgroups fit the 512 columns.
double budgets_for(const int* dps, const double* work, int n_dps, int warpgroups, int* cols) {
    double total = 0.0;
    for (int i = 0; i < n_dps; ++i) total += work[i];
    if (total <= 0.0) total = 1.0;
    double best = 0.0;
    int best_sum = -1;
    int pick[kAggMaxWarpgroups] = {};
    // Non-increasing index sequences pick[0] = 0 <= pick[1] <= ... < n_dps.
    std::function<void(int, int, int)> rec = [&](int w, int lo, int sum) {
        if (sum > 512) return;
        if (w == warpgroups) {
            double ratio = 0.0, cum = 0.0;
            for (int j = 0; j < n_dps; ++j) {
                cum += work[j] / total;
                int n = 0;
                for (int k = 0; k < warpgroups; ++k) n += dps[pick[k]] >= dps[j];
                ratio = std::max(ratio, cum * warpgroups / n);
            }
            if (best_sum < 0 || ratio < best - 1e-9 || (ratio < best + 1e-9 && sum > best_sum)) {
                best = ratio;
                best_sum = sum;
                for (int k = 0; k < warpgroups; ++k) cols[k] = dps[pick[k]];
            }
            return;
        }
        for (int i = lo; i < n_dps; ++i) {
            pick[w] = i;
            rec(w + 1, i, sum + dps[i]);
        }
    };
    if (warpgroups < 1 || warpgroups > kAggMaxWarpgroups || n_dps < 1) return 0.0;
    pick[0] = 0;
    rec(1, 0, dps[0]);
    return best_sum < 0 ? 0.0 : best;
}

int default_warpgroups(const int* dps, const double* work, int n_dps, bool wide_tiles, double path_pd,
                       double chain_steps) {
    // The count whose estimated launch time is lowest. A launch lasts at least
    // as long as its queued work at the rate of w warpgroups an SM, and as long
    // as its longest unit: a serial chain of chain_steps (pixel step x D)
    // updates, slower the more warps share its scheduler. Rates and chain
    // times measured on B200 (148 SMs, 1.965 GHz) with batches of 13 to 64
    // mixed pairs (D 64..192, up to 1920 wide) at each warpgroup count; the
    // work is scaled by budgets_for's ratio when the TMEM budgets of w
    // warpgroups cannot share the work evenly. Four warpgroups (D <= 128
    // only) extrapolate the trend.
    static constexpr double kPathPdPerUs[kAggMaxWarpgroups] = {1.42e6, 2.10e6, 2.32e6, 2.40e6};
    static constexpr double kUsPerChainStep[kAggMaxWarpgroups] = {0.0288, 0.037, 0.045, 0.053};
    const int wmax = max_warpgroups(dps[0], dps[n_dps - 1], wide_tiles);
    int best_w = 1;
    double best_us = 0.0;
    for (int w = 1; w <= wmax; ++w) {
        int cols[kAggMaxWarpgroups];
        const double ratio = budgets_for(dps, work, n_dps, w, cols);
        if (ratio <= 0.0) break;
        const double us = std::max(path_pd * ratio / kPathPdPerUs[w - 1], chain_steps * kUsPerChainStep[w - 1]);
        if (w == 1 || us < best_us) {
            best_us = us;
            best_w = w;
        }
    }
    if (std::getenv("VX_SGM_DEBUG"))
        std::fprintf(stderr, "vx_sgm: %.3g path-pd, longest chain %.3g steps: %d warpgroups (%.0f us estimated)\n",
                     path_pd, chain_steps, best_w, best_us);
    return best_w;
}

static size_t smem_for(int dp_max, bool wide_tiles, int warpgroups) {
    return aggregate_tile_offset(dp_max) + (size_t)warpgroups * 4 * aggregate_warp_smem(dp_max, wide_tiles);
}

cudaError_t prepare() {
    // Dynamic shared memory up to the largest tile area, and the smallest
    // shared-memory carveout: the rest of the SM is L1.
    int dev = 0, max_bytes = 227 * 1024;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&max_bytes, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaError_t e = cudaSuccess;
    for (const void* fn : {aggregate_kernel_fn(false, false), aggregate_kernel_fn(true, false),
                           aggregate_kernel_fn(false, true), aggregate_kernel_fn(true, true)}) {
        cudaFuncAttributes fa{};
        if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, fn);
        if (e == cudaSuccess)   // dynamic + static shared memory must fit the opt-in limit
            e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     max_bytes - (int)fa.sharedSizeBytes);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout,
                                     (int)cudaSharedmemCarveoutMaxL1);
    }
    return e;
}

static int grid_ctas_for() {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms;
}

cudaError_t launch(int dp_max, bool wide_tiles, const AggLaunch& L, const PairDev* d_pairs,
                   const JobDev* d_jobs, const UnitDev* d_units, int num_units, unsigned* counters,
                   cudaStream_t stream, bool compact) {
    if (num_units <= 0) return cudaSuccess;
    const int threads = L.warpgroups * 128;
    const size_t smem = smem_for(dp_max, wide_tiles, L.warpgroups);
    int grid_ctas = grid_ctas_for();
    const int needed = (num_units + threads / 32 - 1) / (threads / 32);
    if (grid_ctas > needed) grid_ctas = needed;
    if (std::getenv("VX_SGM_DEBUG")) {
        std::fprintf(stderr, "vx_sgm: aggregation (pairs) %d CTAs x %d warpgroups, %d TMEM cols, %zu B smem, "
                     "%d queue classes, columns from", grid_ctas, L.warpgroups, L.tmem_cols, smem, L.queues.n_classes);
        for (int w = 0; w < L.warpgroups; ++w)
            std::fprintf(stderr, " %d (class %d)", L.queues.col0[w], L.queues.first_class[w]);
        std::fprintf(stderr, "\n");
    }
    count_launch();
    int tmem_cols = L.tmem_cols;
    AggQueues q = L.queues;
    void* args[] = {&d_pairs, &d_jobs, &d_units, &q, &counters, &dp_max, &tmem_cols};
    return cudaLaunchKernel(aggregate_kernel_fn(wide_tiles, compact), dim3(grid_ctas), dim3(threads),
                            args, smem, stream);
}

}  // namespace pairs

// Both forms, dispatched on the plan's unit size (launch.hpp).
cudaError_t prepare_aggregate_kernels() {
    cudaError_t e = pairs::prepare();
    if (e == cudaSuccess) e = single::prepare();
    return e == cudaSuccess ? prepare_cost_kernels() : e;
}

int aggregate_max_warpgroups(int unit_scanlines, int dp_max, int dp_min, bool census64, bool wide_tiles) {
    if (unit_scanlines == kScanForm) return 1;   // no warpgroup shape: warps per SM by occupancy
    return unit_scanlines == kUnitScanlines ? pairs::max_warpgroups(dp_max, dp_min, wide_tiles)
                                            : single::max_warpgroups(dp_max, census64);
}

cudaError_t launch_aggregate(int unit_scanlines, int dp_max, int dp_min, bool census64, bool wide_tiles, const AggLaunch& L,
                             const PairDev* d_pairs, const JobDev* d_jobs, const UnitDev* d_units,
                             int num_units, unsigned* counters, cudaStream_t stream, bool compact) {
    if (unit_scanlines == kUnitScanlines)
        return pairs::launch(dp_max, wide_tiles, L, d_pairs, d_jobs, d_units, num_units, counters, stream, compact);
    if (unit_scanlines == kScanForm)
        return scan::launch(d_pairs, d_jobs, d_units, num_units, counters, stream, compact);
    return single::launch(dp_max, census64, L.warpgroups, d_pairs, d_jobs, d_units, num_units, counters, stream,
                          compact);
}

}  // namespace vxsgm
