// Launch helpers for the sweep kernels (implemented in sa_launch.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "sa_types.h"

namespace b200sa {

constexpr int kMaxThreadsPerCta = 512;

// Kernel variant: bit 0 Gibbs, bit 1 random order, bit 2 state in shared
// memory.
inline int kernel_variant(bool gibbs, bool random_order, bool smem) {
    return (gibbs ? 1 : 0) | (random_order ? 2 : 0) | (smem ? 4 : 0);
}

cudaError_t upload_jump_table(const uint32_t table[][4], cudaStream_t stream);
cudaError_t launch_sa(int variant, const LaunchArgs &args, int grid, int warps_per_cta,
                      int region_bytes, cudaStream_t stream);
cudaError_t kernel_occupancy(int variant, int warps_per_cta, int region_bytes,
                             int *ctas_per_sm);
cudaError_t acceptance_check(int64_t samples, uint64_t seed, unsigned long long *d_counts);

}  // namespace b200sa
