// Matching-cost volume for the scanline-pair aggregation kernel.
//
// Every path of a pair reads the same cost C(x, y, d) (vx-vision's
// SGMStereo.metal:131-142: popcount of the census XOR, 64 where x - d < 0), so
// a batch that runs the scanline-pair form computes it once per pair into a byte
// volume, pixel-major and d-minor like the path slabs (Dv bytes per pixel, the
// pads d >= D zero): the eight paths then read one byte per disparity instead of
// re-forming it from the census words (two XOR, two popcounts and a pack per two
// scanlines). Costs are at most 64, so a byte holds them.
//
// One CTA per image row of the batch (the WTA kernel's row numbering). A warp
// item is one 16-disparity chunk of 128 pixels, 4 consecutive pixels a lane: the
// lane's quad starts on a 4-word boundary of the census plane, so its 4 left
// words and the 20 right words at x - d (x = its pixels, d = the chunk's 16
// disparities) are 16-byte-aligned vector loads, 64 costs from 6 loads (the
// census planes' guard words keep the reads at either end of the plane in
// bounds). Items go to a shared-memory tile of the pass's vectors, which the
// CTA then writes as one contiguous run of the volume with coalesced 16-byte
// stores. A pass covers as many 128-pixel blocks as fill the 8 warps' last
// round of items best (D = 192: 2 blocks, 24 items), within four CTAs' worth of
// shared memory an SM.
#include <cuda_runtime.h>

#include "kernels.cuh"
#include "launch.hpp"

namespace vxsgm {

namespace {

__device__ __forceinline__ int find_pair_by_row(const PairDev* pairs, int n, int row) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (pairs[mid].row_begin <= row) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ uint32_t popc_xor(uint32_t a, uint32_t b) { return __popc(a ^ b); }
__device__ __forceinline__ uint32_t popc_xor(uint64_t a, uint64_t b) { return __popcll(a ^ b); }

constexpr int kBlockPx = 128;     // pixels of a warp item
constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kTileRows = 132;    // tile rows of a block: pixel p at row (p & 3) * 33 + p / 4

// Tile row stride in 16-byte units: odd, so that 8 lanes storing 16 bytes each
// to consecutive rows hit distinct bank groups.
__host__ __device__ constexpr int tile_stride(int dv) { return (dv / 16) | 1; }
constexpr int kMaxTileBytes = 56 * 1024;   // four CTAs an SM
// Blocks of a pass: the count (1..8) whose nb * chunks items fill the 8 warps'
// last round best (the CTA waits for its slowest warp at the end of a pass),
// the smaller on ties, within kMaxTileBytes of tile.
__host__ __device__ constexpr int blocks_per_pass(int dv) {
    const int chunks = dv / 16;
    int best = 1, best_num = 0, best_den = 1;    // efficiency = items / (8 * rounds)
    for (int nb = 1; nb <= kWarps && nb * kTileRows * tile_stride(dv) * 16 <= kMaxTileBytes; ++nb) {
        const int items = nb * chunks, den = kWarps * ((items + kWarps - 1) / kWarps);
        if (items * best_den > best_num * den) best = nb, best_num = items, best_den = den;
    }
    return best;
}
__host__ __device__ constexpr int tile_units(int dv) { return blocks_per_pass(dv) * kTileRows * tile_stride(dv); }

__device__ __forceinline__ void load4(const uint32_t* p, uint32_t* w) {
    const uint4 q = __ldg(reinterpret_cast<const uint4*>(p));
    w[0] = q.x, w[1] = q.y, w[2] = q.z, w[3] = q.w;
}
__device__ __forceinline__ void load4(const uint64_t* p, uint64_t* w) {
    const ulonglong2 a = __ldg(reinterpret_cast<const ulonglong2*>(p));
    const ulonglong2 b = __ldg(reinterpret_cast<const ulonglong2*>(p) + 1);
    w[0] = a.x, w[1] = a.y, w[2] = b.x, w[3] = b.y;
}

// Costs of pixels x4 + i (i < 4) at disparities d0 + e (e < 16): l = their left
// words, r[j] = right word at x4 - d0 - 16 + j, so pixel i at offset e reads
// r[i - e + 16]. CHECK: offsets past pixel i's left edge (e > n0 + i, n0 = x4 -
// d0) cost 64, offsets at or past D (e >= dmax, dmax = D - d0) are pads (0).
template <bool CHECK, typename CT>
__device__ __forceinline__ void chunk_costs(const CT (&l)[4], const CT (&r)[20], int n0, int dmax, uint4 (&v)[4]) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        uint32_t w[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            uint32_t acc = 0;
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                const int e = 4 * q + b;
                uint32_t c = popc_xor(l[i], r[i - e + 16]);
                if (CHECK) c = e >= dmax ? 0u : (e > n0 + i ? 64u : c);
                acc |= c << (8 * b);
            }
            w[q] = acc;
        }
        v[i] = make_uint4(w[0], w[1], w[2], w[3]);
    }
}

template <typename CT>
__global__ void __launch_bounds__(kThreads, sizeof(CT) == 4 ? 4 : 2) cost_kernel(const PairDev* __restrict__ pairs, int num_pairs) {
    extern __shared__ uint4 tile[];
    const int pi = find_pair_by_row(pairs, num_pairs, blockIdx.x);
    const PairDev& pr = pairs[pi];
    const int y = blockIdx.x - pr.row_begin;
    const int W = pr.width, D = pr.nd, Dv = pr.nd_vec;
    const int chunks = Dv / 16, ts = tile_stride(Dv), nb = blocks_per_pass(Dv), items = nb * chunks;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // i / chunks by a multiply (chunks >= 2): exact for i < 2^18 (here i < 2048).
    const uint32_t magic = chunks > 1 ? 0xFFFFFFFFu / (uint32_t)chunks + 1u : 0u;
    const CT* __restrict__ cl0 = static_cast<const CT*>(pr.census_l);
    const CT* __restrict__ cr0 = static_cast<const CT*>(pr.census_r);
    const ptrdiff_t row0 = (ptrdiff_t)y * W;
    uint8_t* __restrict__ out = pr.costs + (size_t)row0 * Dv;
    // Passes start at the row's first 4-word boundary (x = -3..0 of this row).
    for (int xb = -(int)(row0 & 3); xb < W; xb += nb * kBlockPx) {
        for (int it = warp; it < items; it += kWarps) {
            const int blk = chunks > 1 ? (int)__umulhi((uint32_t)it, magic) : it;
            const int ch = it - blk * chunks;
            const int x4 = xb + blk * kBlockPx + 4 * lane;
            if (x4 >= W) continue;
            const ptrdiff_t a = row0 + x4;                      // a multiple of 4
            CT l[4], r[20];
            load4(cl0 + a, l);
            const CT* rp = cr0 + a - 16 * ch - 16;             // >= plane - 256 words (guard: 352)
#pragma unroll
            for (int k = 0; k < 5; ++k) load4(rp + 4 * k, r + 4 * k);
            uint4 v[4];
            const int n0 = x4 - 16 * ch, dmax = D - 16 * ch;
            if (n0 >= 15 && dmax >= 16)
                chunk_costs<false>(l, r, n0, dmax, v);
            else
                chunk_costs<true>(l, r, n0, dmax, v);
            uint4* trow = tile + (blk * kTileRows + lane) * ts + ch;
#pragma unroll
            for (int i = 0; i < 4; ++i) trow[i * 33 * ts] = v[i];
        }
        __syncthreads();
        // Pixels max(xb, 0) .. min(xb + nb * 128, W) - 1: one contiguous run.
        const int p0 = max(xb, 0) - xb, p1 = min(nb * kBlockPx, W - xb);
        const int n16 = (p1 - p0) * chunks;
        uint4* __restrict__ dst = reinterpret_cast<uint4*>(out + (size_t)(xb + p0) * Dv);
        for (int q = threadIdx.x; q < n16; q += kThreads) {
            const int pq = chunks > 1 ? (int)__umulhi((uint32_t)q, magic) : q;
            const int c = q - pq * chunks, pp = pq + p0;
            const int row = (pp >> 7) * kTileRows + (pp & 3) * 33 + ((pp & (kBlockPx - 1)) >> 2);
            dst[q] = tile[row * ts + c];
        }
        __syncthreads();
    }
}

}  // namespace

cudaError_t prepare_cost_kernels() {
    cudaError_t e = cudaFuncSetAttribute(cost_kernel<uint32_t>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         kMaxTileBytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(cost_kernel<uint64_t>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxTileBytes);
    return e;
}

cudaError_t launch_costs(const PairDev* d_pairs, int num_pairs, int total_rows, int dp_max, bool census64,
                         cudaStream_t stream) {
    if (total_rows == 0) return cudaSuccess;
    int units = 0;                        // the largest tile of any Dv up to the batch's
    for (int dv = 16; dv <= (dp_max + 15) / 16 * 16; dv += 16) units = units > tile_units(dv) ? units : tile_units(dv);
    const size_t smem = (size_t)units * 16;   // <= kMaxTileBytes
    if (census64)
        cost_kernel<uint64_t><<<total_rows, kThreads, smem, stream>>>(d_pairs, num_pairs);
    else
        cost_kernel<uint32_t><<<total_rows, kThreads, smem, stream>>>(d_pairs, num_pairs);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) count_launch();
    return e;
}

}  // namespace vxsgm
