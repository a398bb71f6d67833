// Launch helpers for the sweep kernel (implemented in sa_launch.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "sa_types.h"

namespace b200sa {

constexpr int kMaxThreadsPerCta = 256;

// Per-warp shared region: RNG ring, then delta energies, then spins.
inline int region_bytes_for(int cap_n) {
    const int spins = (cap_n + 15) & ~15;
    return kRing * (int)sizeof(uint64_t) + cap_n * (int)sizeof(double) + spins;
}

cudaError_t upload_jump_columns(const uint32_t cols[128][4], cudaStream_t stream);
cudaError_t launch_sa(const LaunchArgs &args, int grid, int warps_per_cta,
                      int region_bytes, cudaStream_t stream);
cudaError_t kernel_occupancy(int warps_per_cta, int region_bytes, int *ctas_per_sm);

}  // namespace b200sa
