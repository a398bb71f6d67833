// Launch helpers for the sweep kernels (implemented in sa_launch.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "sa_types.h"

namespace b200sa {

constexpr int kMaxThreadsPerCta = 512;
// Register budgets of the sweep kernels (per thread): 128 (launch bounds of
// 512 threads, one CTA), kRegs80 and kRegs64.
constexpr int kRegs80 = 80;
constexpr int kRegs64 = 64;
constexpr int kRegClasses = 3;  // 0: 128, 1: 80, 2: 64

// Kernel kind: bit 0 Gibbs, bit 1 random order, bit 2 in-window resolution
// (sequential order only; ProblemDev::resolve).
constexpr int kKindGibbs = 1;
constexpr int kKindRandom = 2;
constexpr int kKindResolve = 4;
constexpr int kNumKinds = 8;

// Kernel variant: bits 0-2 kind, bits 3-4 state location (kStageGlobal,
// kStageShared, kStageSpins), bits 5-6 register class (0: 128, 1: 80, 2: 64
// registers).
inline int kernel_variant(int kind, int stage, int reg_class = 0) {
    return (kind & (kNumKinds - 1)) | (stage << 3) | (reg_class << 5);
}
inline int variant_reg_class(int variant) { return variant >> 5; }

cudaError_t upload_jump_table(const uint32_t table[][4], cudaStream_t stream);
cudaError_t scatter_weights(double *arena, const int64_t *dst, const int32_t *src, int64_t num_j,
                            int64_t total, const double *J, const double *h,
                            cudaStream_t stream);
cudaError_t launch_sa(int variant, const LaunchArgs &args, int grid, int warps_per_cta,
                      int region_bytes, cudaStream_t stream);
cudaError_t kernel_occupancy(int variant, int warps_per_cta, int region_bytes,
                             int *ctas_per_sm);
cudaError_t launch_sd(bool sparse, bool smem, const SdArgs &args, int grid, int warps_per_cta,
                      int region_bytes, cudaStream_t stream);
cudaError_t sd_occupancy(bool sparse, bool smem, int warps_per_cta, int region_bytes,
                         int *ctas_per_sm);
cudaError_t launch_rmc(bool random_order, int proposal, const RmcArgs &args, int grid,
                       int block, cudaStream_t stream);
cudaError_t launch_pimc(bool chain_update, const PimcArgs &args, int grid, int block,
                        cudaStream_t stream);
cudaError_t acceptance_check(int64_t samples, uint64_t seed, unsigned long long *d_counts);

}  // namespace b200sa
