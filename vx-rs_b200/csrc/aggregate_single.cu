// Path aggregation of semi-global matching, single-scanline form: every path of
// every pair of a batch in ONE persistent launch over a work queue of (pair,
// path, 32-scanline) units, one scanline per thread. Plans with few units (a
// single pair, small served batches) run this form: it has twice as many units
// as the scanline-pair form (aggregate.cu) and half the work per thread, so a
// lone pair finishes sooner; large batches run the scanline-pair form.
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
//     t_d = min(A_d, f_{d-1});  f_d = u16(t_d + C_d + P1 - m);  Lp[d] = u16(t_d + C_d - m)
// whose critical path is one min and one add per disparity. u16 values live in
// the low half of 32-bit registers: min.u16x2 compares halves on their own and a
// 32-bit add's low half is the u16 sum, so whatever accumulates in the high half
// never reaches the low half and no masking is needed. A_d is formed two
// disparities at a time on packed state words (min.u16x2, and a per-half
// wrapping add for Lp[d+1] + P1).
//
// Mapping. One thread owns one scanline. Its D state values (packed u16 pairs)
// live in tensor memory (TMEM): the thread's TMEM lane, one 32-bit column per
// pair, read and written 4 columns (8 disparities) at a time by warp-collective
// tcgen05.ld/st. The per-pixel loop runs over groups of 8 disparities with a
// small loop body and a runtime D, so one kernel serves every D of a batch, and
// shared memory is left almost entirely to L1 for the census windows. A warp takes 32 neighbouring scanlines of
// one (pair, path):
//  * vertical / diagonal paths: the 32 lanes sit on 32 consecutive pixels of one
//    row at every step, so the right-census words they need form one segment of
//    Dp+31 words of that row; it is staged in warp-private shared memory with
//    16-byte cp.async copies one step ahead (double-buffered).
//  * horizontal paths: the 32 lanes are 32 consecutive rows (one 32-row band)
//    at the same x and read the banded census copy: each disparity is one
//    coalesced 128-byte load at a constant offset, and the window of the last D
//    columns stays in L1.
// Census words of the next group are loaded while the current group is
// processed. Pixels whose window may reach x-d < 0 take a second body with the
// border test, picked by a warp-uniform branch. Results leave as 16-byte stores
// into this path's slab, one byte per disparity: the values of a vector are
// bounded by the census cost plus P2 unless the in-place o1 term pulls them
// below m (then they wrap), so almost every vector fits bytes; one that does
// not is marked with 0xFF in byte 0 and written exactly to a u16 shadow slab.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>

#include "kernels.cuh"
#include "launch.hpp"

namespace vxsgm {
namespace single {

namespace {

constexpr unsigned kFull = 0xffffffffu;
// Largest CTA (6 warpgroups); keeps registers per thread <= 85.
constexpr int kMaxThreads = 768;

__device__ __forceinline__ uint32_t vmin2(uint32_t a, uint32_t b) {
    uint32_t r;
    asm("min.u16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}

__device__ __forceinline__ uint32_t vmax2(uint32_t a, uint32_t b) {
    uint32_t r;
    asm("max.u16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}

__device__ __forceinline__ uint32_t popc_xor(uint32_t a, uint32_t b) { return __popc(a ^ b); }
__device__ __forceinline__ uint32_t popc_xor(uint64_t a, uint64_t b) { return __popcll(a ^ b); }

// 16-byte global -> shared copy that bypasses L1 (staged words are used once).
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;"); }
__device__ __forceinline__ void cp_async_wait_1() {
    asm volatile("cp.async.wait_group 1;" ::: "memory");
}

// Tensor-memory (TMEM) access for the per-scanline state. Warp w of the CTA owns
// TMEM lanes 32w..32w+31 (one lane per thread) and the CTA's allocated columns;
// the 8 disparities of group g are columns 4g..4g+3 (one u16 pair per column).
// tcgen05.ld is asynchronous: its registers are threaded through the wait so
// that no use can be scheduled before the data has arrived.
__device__ __forceinline__ uint4 tmem_ld4(uint32_t taddr) {
    uint4 r;
    __syncwarp();  // .sync.aligned: the whole warp, converged
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
                 : "r"(taddr));
    return r;
}
__device__ __forceinline__ void tmem_wait_ld(uint4& r) {
    __syncwarp();
    asm volatile("tcgen05.wait::ld.sync.aligned;" : "+r"(r.x), "+r"(r.y), "+r"(r.z), "+r"(r.w)::"memory");
}
__device__ __forceinline__ void tmem_st4(uint32_t taddr, uint4 v) {
    __syncwarp();
    asm volatile("tcgen05.st.sync.aligned.32x32b.x4.b32 [%0], {%1, %2, %3, %4};" ::"r"(taddr),
                 "r"(v.x), "r"(v.y), "r"(v.z), "r"(v.w)
                 : "memory");
}
__device__ __forceinline__ void tmem_wait_st() {
    __syncwarp();
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}

// Per-scanline constants of one unit.
struct ScanConst {
    uint32_t p1x2;        // P1 in both halves
    uint32_t P1, P2;
    int Dp, G;            // disparities padded to 8, groups of 8
    int last_j;           // position of d = D-1 inside the last group (0..7)
};

// Per-pixel values shared by the groups of one pixel.
struct PixelState {
    uint32_t o3x2;   // u16(m + P2) in both halves
    uint32_t kc;     // f = t + C + (P1 - m)
    uint32_t km;     // Lp = t + C - m
    uint32_t f;      // o1 of the next disparity (low half)
    uint32_t mn;     // running min of the new values (per half)
    uint32_t mx;     // running max of the new values (per half, d < D)
};

// Matching costs of one group from its 8 right-census words; x-d < 0 gives 64.
template <bool CHECK, typename CT>
__device__ __forceinline__ void group_costs(uint32_t (&c)[8], const CT lc, const CT (&r)[8],
                                            const int x, const int g) {
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        c[i] = popc_xor(lc, r[i]);
        if (CHECK && x - (8 * g + i) < 0) c[i] = 64u;
    }
}

// Writes the warp's output tile to a wide (u16) slab: lanes [la, lb] hold the
// results of one pixel step; row p's vector goes to dst0 + p * stride (in u16),
// and 16-byte word g of it to +8g. Words are distributed over the lanes in
// address order, so consecutive lanes write consecutive 16 bytes of a vector.
__device__ __forceinline__ void flush_tile_wide(const uint4* __restrict__ tile, int row_words, int G,
                                                int la, int lb, uint16_t* __restrict__ dst0,
                                                size_t stride, int lane) {
    __syncwarp();
    // Word c = (p - la) * G + g of the run, walked with a running (p, g) so
    // that no division is needed per word: lane starts at c = lane, steps 32.
    const int n = (lb - la + 1) * G;
    const int q = 32 / G, r = 32 % G;
    int p = la + lane / G, g = lane % G;
    for (int c = lane; c < n; c += 32) {
        __stcs(reinterpret_cast<uint4*>(dst0 + (size_t)p * stride + 8 * g), tile[p * row_words + g]);
        g += r;
        p += q;
        if (g >= G) {
            g -= G;
            ++p;
        }
    }
    __syncwarp();
}

// Writes the warp's output tile to the byte slab: lanes [la, lb] hold the
// results of one pixel step; row p's vector goes to dst0 + p * stride bytes,
// its 16-byte chunk h holding d = 16h..16h+15 (tile words 2h and 2h+1, the low
// byte of every u16). A row whose bit is set in em (escaped, pixel pix0 + p *
// pstride) first gets a shadow slot s and its exact u16 words go to
// shadow + s * Dp; then its byte row is written with 0xFF in byte 0 and s in
// bytes 4..7 (the slot is put into the tile words whose low bytes form them).
// Chunks are distributed over the lanes in address order, so that consecutive
// lanes write consecutive 16 bytes of a vector (streaming stores: slabs are
// read once by the WTA kernel and must not push the census planes, which every
// path re-reads, out of L2).
// Without CP (no shadow pool in the batch) the escaped vectors' u16 words go to
// sh0 + p * sstride, their pixels' places in the full shadow, after the chunks.
template <bool CP>
__device__ __forceinline__ void flush_tile(uint4* __restrict__ tile, int row_words, int G, int la, int lb,
                                           unsigned em, uint8_t* __restrict__ dst0, size_t stride,
                                           uint16_t* __restrict__ sh0, size_t sstride, const EscapeTarget& et,
                                           size_t pix0, size_t pstride, int lane) {
    __syncwarp();
    // Escaped vectors (rare): a slot each, their u16 words, the slot into the tile.
    if constexpr (CP) for (unsigned m = em; m; m &= m - 1) {
        const int pe = __ffs(m) - 1;               // bit p of em = row p (la <= p <= lb)
        uint32_t slot = 0;
        if (lane == 0) slot = take_slot(et, pix0 + (size_t)pe * pstride);
        slot = __shfl_sync(kFull, slot, 0);
        if (slot != kNoSlot)
            for (int g = lane; g < G; g += 32)
                __stcs(reinterpret_cast<uint4*>(et.shadow + (size_t)slot * et.Dp + 8 * g), tile[pe * row_words + g]);
        __syncwarp();
        if (lane == 0) {
            tile[pe * row_words].z = (slot & 0xFFu) | ((slot >> 8) & 0xFFu) << 16;
            tile[pe * row_words].w = ((slot >> 16) & 0xFFu) | (slot >> 24) << 16;
        }
        __syncwarp();
    }
    // Chunk c = (p - la) * V + h of the run, walked with a running (p, h) so
    // that no division is needed per chunk: lane starts at c = lane, steps 32.
    const int V = (G + 1) >> 1;
    const int n = (lb - la + 1) * V;
    const int q = 32 / V, r = 32 % V;
    int p = la + lane / V, h = lane % V;
    for (int c = lane; c < n; c += 32) {
        const uint4* row = tile + p * row_words;
        const uint4 a = row[2 * h];
        const uint4 b = 2 * h + 1 < G ? row[2 * h + 1] : make_uint4(0u, 0u, 0u, 0u);
        uint4 o;
        o.x = __byte_perm(a.x, a.y, 0x6420);
        o.y = __byte_perm(a.z, a.w, 0x6420);
        o.z = __byte_perm(b.x, b.y, 0x6420);
        o.w = __byte_perm(b.z, b.w, 0x6420);
        if (h == 0 && ((em >> p) & 1u)) o.x |= 0xFFu;
        __stcs(reinterpret_cast<uint4*>(dst0 + (size_t)p * stride + 16 * h), o);
        h += r;
        p += q;
        if (h >= V) {
            h -= V;
            ++p;
        }
    }
    if constexpr (!CP) {
        // Escaped vectors (rare): the warp writes their u16 words, one row at a time.
        while (em) {
            const int pe = __ffs(em) - 1;          // bit p of em = row p (la <= p <= lb)
            em &= em - 1;
            for (int g = lane; g < G; g += 32)
                __stcs(reinterpret_cast<uint4*>(sh0 + (size_t)pe * sstride + 8 * g), tile[pe * row_words + g]);
        }
    }
    __syncwarp();
}

// One group of 8 disparities d = 8g..8g+7 of one pixel. cur = old state words of
// the group, nxt_lo = old Lp[8g+8] in the low half (unused for the last group),
// c = the group's matching costs. LAST: the group holding d = D-1, whose o2 is
// forced to 0xFFFF and whose pads (d >= D) are kept out of the minimum.
template <bool LAST>
__device__ __forceinline__ uint4 sgm_group(const uint4 cur, const uint32_t nxt_lo,
                                           const uint32_t (&c)[8], const ScanConst& k,
                                           PixelState& ps) {
    const uint32_t w[5] = {cur.x, cur.y, cur.z, cur.w, nxt_lo};
    uint32_t out[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        uint32_t o2 = __vadd2(__byte_perm(w[j], w[j + 1], 0x5432), k.p1x2);
        if (LAST) {
            if (k.last_j == 2 * j) o2 |= 0x0000FFFFu;
            if (k.last_j == 2 * j + 1) o2 |= 0xFFFF0000u;
        }
        const uint32_t A = vmin2(vmin2(w[j], o2), ps.o3x2);
        const uint32_t t0 = vmin2(A, ps.f);
        ps.f = t0 + c[2 * j] + ps.kc;
        const uint32_t e0 = t0 + c[2 * j] + ps.km;
        const uint32_t t1 = vmin2(A >> 16, ps.f);
        ps.f = t1 + c[2 * j + 1] + ps.kc;
        const uint32_t e1 = t1 + c[2 * j + 1] + ps.km;
        out[j] = __byte_perm(e0, e1, 0x5410);
    }
    if (!LAST) {
        ps.mn = vmin2(ps.mn, vmin2(vmin2(out[0], out[1]), vmin2(out[2], out[3])));
        ps.mx = vmax2(ps.mx, vmax2(vmax2(out[0], out[1]), vmax2(out[2], out[3])));
    } else {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            uint32_t pm = out[j], po = out[j];
            if (2 * j > k.last_j) { pm |= 0x0000FFFFu; po &= 0xFFFF0000u; }   // pads never count
            if (2 * j + 1 > k.last_j) { pm |= 0xFFFF0000u; po &= 0x0000FFFFu; }
            ps.mn = vmin2(ps.mn, pm);
            ps.mx = vmax2(ps.mx, po);
        }
    }
    return make_uint4(out[0], out[1], out[2], out[3]);
}

// One pixel of the 32 scanlines of a warp (all lanes execute it: the TMEM
// accesses are warp-collective). tstate = this warp's TMEM address (lane field
// = its first lane, column 0). getR(d) = right census at x-d; only called with
// x-d >= 0 when CHECK. active: this lane's scanline covers the pixel; an idle lane keeps (or
// resets to) the zero state a scanline starts from. otile = this lane's row of
// the warp's shared-memory output tile (one 16-byte word per group). Returns
// whether the new vector escapes the byte slab. Software pipeline over groups
// (loop unrolled by two, register sets in ping-pong): while group g runs its
// min/add chain, the census words and state of group g+1 are in flight, and
// g+1's costs are formed right after g's chain, so neither load nor popcount
// latency sits on the chain.
template <bool CHECK, typename CT, typename GetR>
__device__ __forceinline__ bool sgm_pixel(const uint32_t tstate, uint32_t& m, const CT lc,
                                          const GetR& getR, const int x, const bool active,
                                          const ScanConst& k,
                                          uint4* __restrict__ otile) {
    PixelState ps;
    const uint32_t o3 = (m + k.P2) & 0xFFFFu;
    ps.o3x2 = o3 | (o3 << 16);
    ps.kc = k.P1 - m;
    ps.km = 0u - m;
    ps.f = 0xFFFFu;            // o1 at d = 0
    ps.mn = 0xFFFFFFFFu;
    ps.mx = 0u;
    auto load = [&](CT (&r)[8], int g) {
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int d = 8 * g + i;
            r[i] = (!CHECK || x - d >= 0) ? getR(d) : CT(0);
        }
    };
    // Results go to this lane's row of the warp's output tile (written to the
    // slab, coalesced, by flush_tile); idle lanes keep a zero state.
    auto store = [&](uint4 o, int g) {
        otile[g] = o;
        if (!active) o = make_uint4(0u, 0u, 0u, 0u);
        tmem_st4(tstate + 4 * g, o);
    };
    CT ra[8], rb[8];
    uint32_t ca[8], cb[8];
    load(ra, 0);
    uint4 sa = tmem_ld4(tstate), sb;
    group_costs<CHECK>(ca, lc, ra, x, 0);
    tmem_wait_ld(sa);
    int g = 0;
#pragma unroll 1
    for (; g + 2 < k.G; g += 2) {
        sb = tmem_ld4(tstate + 4 * (g + 1));
        load(rb, g + 1);
        tmem_wait_ld(sb);
        store(sgm_group<false>(sa, sb.x, ca, k, ps), g);
        group_costs<CHECK>(cb, lc, rb, x, g + 1);
        sa = tmem_ld4(tstate + 4 * (g + 2));
        load(ra, g + 2);
        tmem_wait_ld(sa);
        store(sgm_group<false>(sb, sa.x, cb, k, ps), g + 1);
        group_costs<CHECK>(ca, lc, ra, x, g + 2);
    }
    if (g + 1 < k.G) {
        sb = tmem_ld4(tstate + 4 * (g + 1));
        load(rb, g + 1);
        tmem_wait_ld(sb);
        store(sgm_group<false>(sa, sb.x, ca, k, ps), g);
        group_costs<CHECK>(cb, lc, rb, x, g + 1);
        store(sgm_group<true>(sb, 0u, cb, k, ps), g + 1);
    } else {
        store(sgm_group<true>(sa, 0u, ca, k, ps), g);
    }
    tmem_wait_st();            // the next pixel reads this state back
    m = active ? min(ps.mn & 0xFFFFu, ps.mn >> 16) : 0u;
    // The vector escapes the byte slab when a value is 255 or more, so that a
    // stored byte vector never holds the marker 0xFF.
    return max(ps.mx & 0xFFFFu, ps.mx >> 16) >= 0xFFu;
}

__device__ __forceinline__ ScanConst scan_const(const PairDev& pr) {
    ScanConst k;
    k.P1 = (uint32_t)pr.p1;
    k.P2 = (uint32_t)pr.p2;
    k.p1x2 = k.P1 | (k.P1 << 16);
    k.Dp = pr.nd_pad;
    k.G = pr.nd_pad / 8;
    k.last_j = (pr.nd - 1) - 8 * (k.G - 1);
    return k;
}

__device__ __forceinline__ void clear_state(uint32_t tstate, int G) {
    for (int g = 0; g < G; ++g) tmem_st4(tstate + 4 * g, make_uint4(0u, 0u, 0u, 0u));
    tmem_wait_st();
}

// Unit = 32 scanlines of a vertical or diagonal path.
template <typename CT, bool CP>
__device__ __forceinline__ void run_vertical_unit(const PairDev& pr, const JobDev& job, int first,
                                                  uint32_t tstate, CT* __restrict__ stage,
                                                  int seg_words, uint4* __restrict__ tile,
                                                  int row_words) {
    const int lane = threadIdx.x & 31;
    const int W = pr.width, H = pr.height;
    const ScanConst k = scan_const(pr);
    const int Dp = k.Dp;
    const int dx = job.dx, dy = job.dy;

    const int i = first + lane;
    const int k0 = job.k_min + first;         // scanline index of lane 0
    const int kk = k0 + lane;
    // Lane pixel at step t: x = kk + dx*t, y = y0 + dy*t (vertical: dx = 0).
    const int y0 = dy > 0 ? 0 : H - 1;
    int tb, te;
    if (dx == 0) { tb = 0; te = H; }
    else if (dx > 0) { tb = max(0, -kk); te = min(H, W - kk); }
    else { tb = max(0, kk - W + 1); te = min(H, kk + 1); }
    if (i >= job.num_scanlines) { tb = 0x7fffffff; te = -1; }
    const int t_lo = __reduce_min_sync(kFull, tb);
    const int t_hi = __reduce_max_sync(kFull, te);
    if (t_lo >= t_hi) return;

    const CT* __restrict__ CL = static_cast<const CT*>(pr.census_l);
    const CT* __restrict__ CR = static_cast<const CT*>(pr.census_r);
    uint8_t* __restrict__ out = pr.slabs + pr.slab_stride * (size_t)job.path;
    uint16_t* __restrict__ shd = pr.shadow + pr.shadow_stride * (size_t)job.path;
    const EscapeTarget et = CP ? escape_target(pr, job.path) : EscapeTarget{};
    const int Dv = pr.nd_vec;

    // Stage the right-census segment [xb-(Dp-1), xb+31] of the step's row in
    // 16-byte chunks from the aligned word at or below its start. The planes are
    // surrounded by guard words (kCensusGuardWords), so the chunks may run past
    // the row ends: words outside the image are never used for a cost (lanes
    // with x >= W are idle and x-d < 0 takes the border body).
    // The alignment is taken on the plane's linear word index (row starts y*W
    // are not 16-byte aligned in general); the plane base is.
    constexpr int kPerChunk = 16 / sizeof(CT);
    auto seg_start = [&](int t) {
        return (ptrdiff_t)(y0 + dy * t) * W + (k0 + dx * t - (Dp - 1));
    };
    auto stage_step = [&](int t, int buf) {
        const ptrdiff_t ls = seg_start(t);
        const ptrdiff_t la = ls & ~(ptrdiff_t)(kPerChunk - 1);
        const CT* src = CR + la;
        CT* dstb = stage + buf * seg_words;
        const int chunks = (Dp + 31 + (int)(ls - la) + kPerChunk - 1) / kPerChunk;
        for (int j = lane; j < chunks; j += 32) cp_async16(dstb + j * kPerChunk, src + j * kPerChunk);
        cp_async_commit();
    };
    auto seg_offset = [&](int t) {
        const ptrdiff_t ls = seg_start(t);
        return (int)(ls - (ls & ~(ptrdiff_t)(kPerChunk - 1)));
    };

    clear_state(tstate, k.G);
    uint32_t m = 0u;
    stage_step(t_lo, t_lo & 1);
    CT lc_next = CT(0);
    if (t_lo >= tb && t_lo < te) lc_next = CL[(size_t)(y0 + dy * t_lo) * W + kk + dx * t_lo];
    for (int t = t_lo; t < t_hi; ++t) {
        if (t + 1 < t_hi) stage_step(t + 1, (t + 1) & 1);
        else cp_async_commit();                 // keep one group per step
        const CT lc = lc_next;
        const bool active = t >= tb && t < te;
        const int x = kk + dx * t;
        const int y = y0 + dy * t;
        if (t + 1 < t_hi && t + 1 >= tb && t + 1 < te)
            lc_next = CL[(size_t)(y + dy) * W + (x + dx)];
        cp_async_wait_1();
        __syncwarp();
        const CT* seg = stage + (t & 1) * seg_words + seg_offset(t) + lane + (Dp - 1);  // seg[-d] = R(x-d)
        auto getR = [seg](int d) { return seg[-d]; };
        const int xb = k0 + dx * t;             // smallest x of the warp
        uint4* otile = tile + lane * row_words;
        const bool esc = xb >= Dp - 1
                             ? sgm_pixel<false, CT>(tstate, m, lc, getR, x, active, k, otile)
                             : sgm_pixel<true, CT>(tstate, m, lc, getR, x, active, k, otile);
        // Active lanes are one run of consecutive pixels of row y.
        const unsigned act = __ballot_sync(kFull, active);
        const unsigned em = __ballot_sync(kFull, active && esc);
        if (act) {
            const int la = __ffs(act) - 1, lb = 31 - __clz(act);
            const size_t pix0 = (size_t)y * W + xb;
            if (pr.wide_slabs)
                flush_tile_wide(tile, row_words, k.G, la, lb, shd + pix0 * Dp, (size_t)Dp, lane);
            else
                flush_tile<CP>(tile, row_words, k.G, la, lb, em, out + pix0 * Dv, (size_t)Dv, shd + pix0 * Dp,
                               (size_t)Dp, et, pix0, 1, lane);
        }
        __syncwarp();
    }
}

// Unit = 32 rows of a horizontal path (column-major census).
template <typename CT, bool CP>
__device__ __forceinline__ void run_horizontal_unit(const PairDev& pr, const JobDev& job,
                                                    int first, uint32_t tstate,
                                                    uint4* __restrict__ tile, int row_words) {
    const int lane = threadIdx.x & 31;
    const int W = pr.width, H = pr.height;
    const ScanConst k = scan_const(pr);
    const int Dp = k.Dp;
    const int dx = job.dx;
    const int y = first + lane;                 // row of this lane
    const bool active = y < job.num_scanlines;
    const int nrows = min(32, job.num_scanlines - first);
    // Banded census: word (x, y) at ((y / 32) * W + x) * 32 + y % 32, so the 32
    // rows of this unit (first is a multiple of 32) read 128 contiguous bytes per
    // column and column x-d sits at a constant offset of -32*d words. Bands are
    // allocated whole, so idle lanes (rows >= H) read allocated words.
    const size_t band = (size_t)(first >> 5) * W;
    const CT* __restrict__ CL = static_cast<const CT*>(pr.census_lt) + band * 32 + lane;
    const CT* __restrict__ CR = static_cast<const CT*>(pr.census_rt) + band * 32 + lane;
    uint8_t* __restrict__ out = pr.slabs + pr.slab_stride * (size_t)job.path;
    uint16_t* __restrict__ shd = pr.shadow + pr.shadow_stride * (size_t)job.path;
    const EscapeTarget et = CP ? escape_target(pr, job.path) : EscapeTarget{};
    const int Dv = pr.nd_vec;
    (void)H;

    clear_state(tstate, k.G);
    uint32_t m = 0u;
    const int x0 = dx > 0 ? 0 : W - 1;
    CT lc_next = CL[(size_t)x0 * 32];
    for (int t = 0; t < W; ++t) {
        const int x = x0 + dx * t;
        const CT lc = lc_next;
        if (t + 1 < W) lc_next = CL[(size_t)(x + dx) * 32];
        const CT* col = CR + (size_t)x * 32;        // col[-32*d] = R(x-d, y)
        auto getR = [col](int d) { return col[-32 * d]; };
        uint4* otile = tile + lane * row_words;
        const bool esc = x >= Dp - 1
                             ? sgm_pixel<false, CT>(tstate, m, lc, getR, x, active, k, otile)
                             : sgm_pixel<true, CT>(tstate, m, lc, getR, x, active, k, otile);
        const unsigned em = __ballot_sync(kFull, active && esc);
        // Rows first..first+nrows-1, one vector per row at column x.
        const size_t pix0 = (size_t)first * W + x;
        if (pr.wide_slabs)
            flush_tile_wide(tile, row_words, k.G, 0, nrows - 1, shd + pix0 * Dp, (size_t)W * Dp, lane);
        else
            flush_tile<CP>(tile, row_words, k.G, 0, nrows - 1, em, out + pix0 * Dv, (size_t)W * Dv, shd + pix0 * Dp,
                           (size_t)W * Dp, et, pix0, (size_t)W, lane);
    }
}

// Shared memory per warp: the census staging buffers (2 x (Dp+40) words) and
// the output tile (32 rows of Dp/8 + 1 16-byte words; the pad word keeps the
// rows' 16-byte stores on distinct banks).
__host__ __device__ constexpr size_t single_warp_smem(int dp_max, size_t ct) {
    return 2 * (size_t)(dp_max + 40) * ct + (size_t)32 * (dp_max / 8 + 1) * 16;
}

template <typename CT, bool CP>
__global__ void __launch_bounds__(kMaxThreads)
aggregate_kernel(const PairDev* __restrict__ pairs, const JobDev* __restrict__ jobs,
                 const UnitDev* __restrict__ units, int num_units, unsigned* __restrict__ counter,
                 int dp_max, int tmem_cols, int wg_cols) {
    extern __shared__ __align__(16) unsigned char agg_smem[];
    __shared__ uint32_t tmem_base;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int seg_words = dp_max + 40;                          // Dp+31 words + alignment
    const int row_words = dp_max / 8 + 1;                       // tile row: Dp/8 words + pad
    unsigned char* wbase = agg_smem + (size_t)warp * single_warp_smem(dp_max, sizeof(CT));
    CT* stage = reinterpret_cast<CT*>(wbase);
    uint4* tile = reinterpret_cast<uint4*>(wbase + 2 * seg_words * sizeof(CT));

    // TMEM for the state of all the CTA's scanlines, allocated by warp 0 for the
    // whole persistent loop and released by warp 0 after every warp is done.
    // Warp w owns TMEM lanes 32*(w%4).. (its lane quarter) and, inside them, the
    // columns of its warpgroup w/4: [ (w/4)*wg_cols, (w/4+1)*wg_cols ).
    if (warp == 0) {
        const unsigned slot = (unsigned)__cvta_generic_to_shared(&tmem_base);
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot),
                     "r"(tmem_cols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tstate =
        tmem_base + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)((warp >> 2) * wg_cols);

    for (;;) {
        int u = 0;
        if (lane == 0) u = (int)atomicAdd(counter, 1u);
        u = __shfl_sync(kFull, u, 0);
        if (u >= num_units) break;
        const UnitDev unit = units[u];
        const JobDev job = jobs[unit.job];
        const PairDev& pr = pairs[job.pair];
        if (job.dy == 0)
            run_horizontal_unit<CT, CP>(pr, job, unit.first_scanline, tstate, tile, row_words);
        else
            run_vertical_unit<CT, CP>(pr, job, unit.first_scanline, tstate, stage, seg_words, tile,
                                  row_words);
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

}  // namespace

// Launch shape of the aggregation kernel for a batch whose largest padded D is
// dp_max: one CTA per SM (the CUDA occupancy calculator allows one CTA per SM
// for a kernel that allocates tensor memory) with as many warpgroups as the
// SM's 512 TMEM columns and registers hold. A warpgroup's 4 warps cover the
// 128 TMEM lanes and need dp_max/2 columns.
struct AggShape {
    int warpgroups;
    int wg_cols;     // columns per warpgroup
    int tmem_cols;   // allocation (power of two >= warpgroups * wg_cols)
    size_t smem;     // census staging
};

// Largest number of warpgroups one aggregation CTA can hold for this batch:
// bounded by the 512 TMEM columns, the registers and the shared memory of an SM.
int max_warpgroups(int dp_max, bool census64) {
    const int wg_cols = dp_max / 2;
    const int by_tmem = 512 / wg_cols;
    int regs = 80, regs_sm = 65536, dev = 0, smem_sm = 227 * 1024;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev);
    cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    // Either shadow kind may run with the shape chosen here: the larger register count counts.
    for (bool compact : {false, true}) {
        cudaFuncAttributes fa{};
        const void* fn = census64 ? (compact ? (const void*)aggregate_kernel<uint64_t, true>
                                             : (const void*)aggregate_kernel<uint64_t, false>)
                                  : (compact ? (const void*)aggregate_kernel<uint32_t, true>
                                             : (const void*)aggregate_kernel<uint32_t, false>);
        if (cudaFuncGetAttributes(&fa, fn) == cudaSuccess && fa.numRegs > 0)
            regs = compact ? std::max(regs, fa.numRegs) : fa.numRegs;
    }
    cudaGetLastError();
    const int by_regs = regs_sm / (regs * 128);
    const int by_smem = (int)((smem_sm - 1024) / (4 * single_warp_smem(dp_max, census64 ? 8 : 4)));
    return std::max(1, std::min({by_tmem, by_regs, by_smem, kMaxThreads / 128}));
}

int default_warpgroups(int dp_max, bool census64, int num_units) {
    // Most warpgroups that still leave every warp ~2.5 units of the queue: a
    // scanline is serial work, so a crowded SM slows the longest units down and
    // few units per warp cannot even that out.
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int wmax = max_warpgroups(dp_max, census64);
    int w = 1;
    while (w < wmax && (double)num_units >= 2.5 * sms * 4 * (w + 1)) ++w;
    return w;
}

static AggShape shape_for(int dp_max, bool census64, int warpgroups) {
    AggShape sh{};
    sh.wg_cols = dp_max / 2;
    const int wmax = max_warpgroups(dp_max, census64);
    sh.warpgroups = std::max(1, std::min(warpgroups, wmax));
    sh.tmem_cols = 32;
    while (sh.tmem_cols < sh.warpgroups * sh.wg_cols) sh.tmem_cols <<= 1;
    sh.smem = (size_t)sh.warpgroups * 4 * single_warp_smem(dp_max, census64 ? 8 : 4);
    return sh;
}

cudaError_t prepare() {
    // Dynamic shared memory up to the largest staging area, and the smallest
    // shared-memory carveout: the rest of the SM's L1 caches the census windows.
    int dev = 0, max_bytes = 227 * 1024;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&max_bytes, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaError_t e = cudaSuccess;
    for (const void* fn : {(const void*)aggregate_kernel<uint32_t, false>, (const void*)aggregate_kernel<uint64_t, false>,
                           (const void*)aggregate_kernel<uint32_t, true>, (const void*)aggregate_kernel<uint64_t, true>}) {
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

static int grid_ctas_for(int dp_max, bool census64) {
    (void)dp_max;
    (void)census64;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms;
}

cudaError_t launch(int dp_max, bool census64, int warpgroups, const PairDev* d_pairs,
                             const JobDev* d_jobs, const UnitDev* d_units, int num_units,
                             unsigned* counter, cudaStream_t stream, bool compact) {
    if (num_units <= 0) return cudaSuccess;
    if (warpgroups <= 0) warpgroups = default_warpgroups(dp_max, census64, num_units);
    const AggShape sh = shape_for(dp_max, census64, warpgroups);
    const int threads = sh.warpgroups * 128;
    int grid_ctas = grid_ctas_for(dp_max, census64);
    const int needed = (num_units + threads / 32 - 1) / (threads / 32);
    if (grid_ctas > needed) grid_ctas = needed;
    if (std::getenv("VX_SGM_DEBUG"))
        std::fprintf(stderr, "vx_sgm: aggregation (single) %d CTAs x %d warpgroups, %d TMEM cols, %zu B smem\n",
                     grid_ctas, sh.warpgroups, sh.tmem_cols, sh.smem);
    count_launch();
    auto fn = census64 ? (compact ? aggregate_kernel<uint64_t, true> : aggregate_kernel<uint64_t, false>)
                       : (compact ? aggregate_kernel<uint32_t, true> : aggregate_kernel<uint32_t, false>);
    fn<<<grid_ctas, threads, sh.smem, stream>>>(d_pairs, d_jobs, d_units, num_units, counter, dp_max, sh.tmem_cols,
                                                sh.wg_cols);
    return cudaGetLastError();
}

}  // namespace single
}  // namespace vxsgm
