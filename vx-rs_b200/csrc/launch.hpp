// Host-side launchers of the SGM kernels (implemented in the .cu files).
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>

#include "kernels.cuh"

namespace vxsgm {

// Kernel launches issued by this library since load (bench/test evidence).
extern std::atomic<uint64_t> g_kernel_launches;
inline void count_launch(uint64_t n = 1) { g_kernel_launches.fetch_add(n, std::memory_order_relaxed); }

// Census of both views of every pair: one CTA per 32x8 tile.
cudaError_t launch_census(const PairDev* d_pairs, int num_pairs, int total_tiles, int max_rx,
                          int max_ry, bool census64, cudaStream_t stream);

// Kernel variant of the path aggregation, chosen per group of units.
struct AggVariant {
    int dmax;     // register capacity in disparities: 64, 128, 192, 256
    bool exact;   // D == dmax for every pair of the group
    bool census64;
    bool horizontal;
    bool operator==(const AggVariant& o) const {
        return dmax == o.dmax && exact == o.exact && census64 == o.census64 &&
               horizontal == o.horizontal;
    }
};

// Persistent launch over `num_units` warp units; warps pull units from
// `*counter` (must be zero on entry). grid_ctas = 0 picks SMs x occupancy.
cudaError_t launch_aggregate(const AggVariant& v, const PairDev* d_pairs, const JobDev* d_jobs,
                             const UnitDev* d_units, int num_units, unsigned* counter,
                             int grid_ctas, cudaStream_t stream);

// Number of CTAs a persistent aggregation launch uses for this variant.
int aggregate_grid_ctas(const AggVariant& v);

// WTA + subpixel + optional LR check: one CTA per (pair, row). The kernel keeps
// three words per pixel of the row in shared memory.
size_t wta_smem_bytes(int max_width);
// Raises the kernel's dynamic shared-memory limit; once per device.
cudaError_t prepare_wta_kernel();
cudaError_t launch_wta(const PairDev* d_pairs, int num_pairs, int total_rows, int max_width,
                       cudaStream_t stream);

}  // namespace vxsgm
