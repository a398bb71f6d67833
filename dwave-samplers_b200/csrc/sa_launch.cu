// Kernel entry points: warps take (problem, read) work items, either from a
// device work-queue head (persistent mode: one launch per bucket) or by a
// static stride (plain mode: one launch per problem).  One instantiation per
// acceptance rule, update order and state location, so each keeps only its
// own path's registers, and per register budget: 128 registers a thread (at
// most 16 warps per SM), 80 (24 warps) or 64 (32 warps).  Fewer registers
// mean more spills but more reads in flight per SM, which pays when a bucket
// has enough reads to fill them; the autotuner chooses per bucket.
#include <cuda_runtime.h>

#include <algorithm>

#include "sa_kernel.cuh"
#include "sa_launch.h"
#include "sd_kernel.cuh"
#include "rmc_kernel.cuh"
#include "pimc_kernel.cuh"

namespace b200sa {

template <bool GIBBS, bool RANDOM_ORDER, bool RESOLVE, int STAGE>
__device__ __forceinline__ void sa_warp_body(const LaunchArgs &A, int warps_per_cta,
                                             int region_bytes) {
    extern __shared__ __align__(16) uint8_t smem[];
    const unsigned lane = threadIdx.x & 31u;
    const int wid = (int)(threadIdx.x >> 5);
    uint8_t *region = smem + (size_t)wid * (size_t)region_bytes;
    uint64_t *ring = reinterpret_cast<uint64_t *>(region);
    double *scratch = reinterpret_cast<double *>(region + kRing * sizeof(uint64_t));
    const int64_t gw = (int64_t)blockIdx.x * warps_per_cta + wid;
    const int64_t total_warps = (int64_t)gridDim.x * warps_per_cta;
    double *de;
    int8_t *sp;
    uint32_t *touch = reinterpret_cast<uint32_t *>(region + kRing * sizeof(uint64_t) + kScratchBytes);
    uint8_t *state = region + kRing * sizeof(uint64_t) + kScratchBytes + A.touch_bytes;
    double *band = nullptr;
    if constexpr (STAGE == kStageShared) {
        de = reinterpret_cast<double *>(state);
        sp = reinterpret_cast<int8_t *>(state + (size_t)A.smem_cap_n * sizeof(double));
    } else if constexpr (STAGE == kStageSpins || STAGE == kStageBand) {
        de = A.scratch_de + gw * A.scratch_stride;
        sp = reinterpret_cast<int8_t *>(state);
        if constexpr (STAGE == kStageBand)
            band = reinterpret_cast<double *>(state + (((size_t)A.smem_cap_n + 15) & ~size_t(15)));
    } else {
        de = A.scratch_de + gw * A.scratch_stride;
        sp = A.scratch_s + gw * A.scratch_stride;
    }
    if (A.shared_stream && gw != 0) return;
    if (RANDOM_ORDER) {  // the touch bitmap starts clear; every pass clears what it sets
        for (int i = (int)lane; i < A.touch_bytes / 4; i += 32) touch[i] = 0u;
        __syncwarp();
    }

    RingState rs;
    bool stream_live = false;
    if (A.shared_stream && A.carry_in) {
        for (int i = lane; i < kRing; i += 32) ring[i] = A.rng_carry[i];
        warp_cold(ring)->seg[2 * lane] = A.rng_carry[kRing + 2 * lane];
        warp_cold(ring)->seg[2 * lane + 1] = A.rng_carry[kRing + 2 * lane + 1];
        rs.q = (uint32_t)A.rng_carry[kRing + kCarryLaneWords];
        rs.base = (uint32_t)A.rng_carry[kRing + kCarryLaneWords + 1];
        stream_live = true;
        __syncwarp();
    }

    int64_t it = gw;
    for (;;) {
        if (A.queue_head) {
            unsigned long long x = 0;
            if (lane == 0) x = atomicAdd(A.queue_head, 1ull);
            it = (int64_t)__shfl_sync(kFull, x, 0);
        }
        if (it >= A.num_items) break;
        const int64_t item = A.items[it];
        const int pi = (int)(item >> 32);
        const int r = (int)(item & 0xffffffffll);
        const ProblemDev *PD = &A.problems[pi];
        const int64_t rd = PD->read_offset + r;
        if (!stream_live) {
            ring_init(ring, rs, A.seeds[rd], lane);
            stream_live = A.shared_stream != 0;
        }
        const int64_t so = PD->state_offset + (int64_t)r * PD->n;
        WarpCold *cold = warp_cold(ring);
        if (lane == 0) cold->flips = 0ull, cold->passes = 0ull, cold->near = 0u;
        anneal_read<GIBBS, RANDOM_ORDER, RESOLVE, STAGE>(
            PD, A.states_in + so, A.states_out + so, &A.energies[rd], de, sp, scratch, ring, rs,
            lane, touch, band, A.band_cap);
        if (lane == 0) {
            A.stats[rd].flips = cold->flips;
            A.stats[rd].passes = cold->passes;
            A.stats[rd].near_ties = cold->near;
        }
        if (!A.queue_head) it += A.shared_stream ? 1 : total_warps;
    }

    if (A.shared_stream && stream_live) {
        __syncwarp();
        for (int i = lane; i < kRing; i += 32) A.rng_carry[i] = ring[i];
        A.rng_carry[kRing + 2 * lane] = warp_cold(ring)->seg[2 * lane];
        A.rng_carry[kRing + 2 * lane + 1] = warp_cold(ring)->seg[2 * lane + 1];
        if (lane == 0) {
            A.rng_carry[kRing + kCarryLaneWords] = rs.q;
            A.rng_carry[kRing + kCarryLaneWords + 1] = rs.base;
        }
    }
}

template <bool GIBBS, bool RANDOM_ORDER, bool RESOLVE, int STAGE>
__global__ void __launch_bounds__(kMaxThreadsPerCta, 1)
    sa_warp_kernel(LaunchArgs A, int warps_per_cta, int region_bytes) {
    sa_warp_body<GIBBS, RANDOM_ORDER, RESOLVE, STAGE>(A, warps_per_cta, region_bytes);
}

template <bool GIBBS, bool RANDOM_ORDER, bool RESOLVE, int STAGE>
__global__ void __maxnreg__(kRegs80) sa_warp_kernel_r80(LaunchArgs A, int warps_per_cta,
                                                         int region_bytes) {
    sa_warp_body<GIBBS, RANDOM_ORDER, RESOLVE, STAGE>(A, warps_per_cta, region_bytes);
}

template <bool GIBBS, bool RANDOM_ORDER, bool RESOLVE, int STAGE>
__global__ void __maxnreg__(kRegs64) sa_warp_kernel_r64(LaunchArgs A, int warps_per_cta,
                                                         int region_bytes) {
    sa_warp_body<GIBBS, RANDOM_ORDER, RESOLVE, STAGE>(A, warps_per_cta, region_bytes);
}

using KernelFn = void (*)(LaunchArgs, int, int);

// Kinds in the order of their numbers (bit 0 Gibbs, bit 1 random order,
// bit 2 in-window resolution); resolution exists for sequential order only.
#define B200SA_KINDS(name, stage)                                                      \
    name<false, false, false, stage>, name<true, false, false, stage>,                 \
        name<false, true, false, stage>, name<true, true, false, stage>,               \
        name<false, false, true, stage>, name<true, false, true, stage>, nullptr, nullptr
// The band location exists for sequential order only.
#define B200SA_SEQ_KINDS(name, stage)                                                  \
    name<false, false, false, stage>, name<true, false, false, stage>, nullptr, nullptr, \
        name<false, false, true, stage>, name<true, false, true, stage>, nullptr, nullptr
#define B200SA_KERNEL_TABLE(name)                                                      \
    {B200SA_KINDS(name, kStageGlobal), B200SA_KINDS(name, kStageShared),              \
     B200SA_KINDS(name, kStageSpins), B200SA_SEQ_KINDS(name, kStageBand)}

static KernelFn kernel_for(int variant) {
    constexpr int kPerClass = kNumStages * kNumKinds;
    static const KernelFn k128[kPerClass] = B200SA_KERNEL_TABLE(sa_warp_kernel);
    static const KernelFn k80[kPerClass] = B200SA_KERNEL_TABLE(sa_warp_kernel_r80);
    static const KernelFn k64[kPerClass] = B200SA_KERNEL_TABLE(sa_warp_kernel_r64);
    const int idx = variant & 31;  // kind (bits 0-2) and state location (bits 3-4)
    if (idx >= kPerClass) return nullptr;
    switch (variant_reg_class(variant)) {
        case 0: return k128[idx];
        case 1: return k80[idx];
        case 2: return k64[idx];
        default: return nullptr;
    }
}

// Diagnostic: compares the single-precision acceptance bounds with the exact
// double-precision decisions on pseudo-random arguments, half of them placed
// within 2^-8 (relative) of the decision boundary.  counts[0..5] =
// Metropolis {samples, decided fast, fast disagreeing with exact},
// Gibbs {samples, decided fast, fast disagreeing with exact}.
__global__ void acceptance_check_kernel(int64_t samples, uint64_t seed,
                                        unsigned long long *counts) {
    uint64_t s0 = seed ^ (0x9e3779b97f4a7c15ull * (blockIdx.x * blockDim.x + threadIdx.x + 1));
    uint64_t s1 = 0x2545f4914f6cdd1dull;
    for (int i = 0; i < 20; ++i) xs_next(s0, s1);
    unsigned long long mf = 0, mx = 0, gf = 0, gx = 0, nm = 0, ng = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < samples;
         i += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t a = xs_next(s0, s1), b = xs_next(s0, s1), c = xs_next(s0, s1);
        const double u = (double)(a >> 11) * 0x1p-53;           // [0, 1)
        const double eps = ((double)(c >> 11) * 0x1p-53 - 0.5) * 0x1p-7;
        {  // Metropolis: x in (-44.4, 0]
            const double x = -44.4 * u;
            uint64_t r = b;
            if (i & 1) {
                const double t = exp(x) * kTwo64 * (1.0 + eps);
                r = t >= kTwo64 ? ~0ull : (uint64_t)t;
            }
            const bool exact = exp(x) * kTwo64 > __ull2double_rn(r);
            const int f = metropolis_fast(x, r);
            ++nm;
            if (f >= 0) {
                ++mf;
                if ((f != 0) != exact) ++mx;
            }
        }
        {  // Gibbs: z in (-60, 44.4)
            const double z = -60.0 + 104.4 * u;
            uint64_t r = b;
            if (i & 1) {
                const double t = kTwo64 / (1.0 + exp(z)) * (1.0 + eps);
                r = t >= kTwo64 ? ~0ull : (uint64_t)t;
            }
            const bool exact = kTwo64 > __ull2double_rn(r) * (1.0 + exp(z));
            const int f = gibbs_fast(z, r);
            ++ng;
            if (f >= 0) {
                ++gf;
                if ((f != 0) != exact) ++gx;
            }
        }
    }
    atomicAdd(&counts[0], nm);
    atomicAdd(&counts[1], mf);
    atomicAdd(&counts[2], mx);
    atomicAdd(&counts[3], ng);
    atomicAdd(&counts[4], gf);
    atomicAdd(&counts[5], gx);
}

cudaError_t acceptance_check(int64_t samples, uint64_t seed, unsigned long long *d_counts) {
    acceptance_check_kernel<<<148 * 4, 256>>>(samples, seed, d_counts);
    return cudaGetLastError();
}

// arena[dst[i]] = (i < num_j ? J[src[i]] : h[src[i]]): the coupler weights
// (adjacency entries, COO copy, back-neighbour copies) and the fields of
// every problem of a plan, from the concatenated inputs.
__global__ void scatter_weights_kernel(double *arena, const int64_t *dst, const int32_t *src,
                                       int64_t num_j, int64_t total, const double *J,
                                       const double *h) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x)
        arena[dst[i]] = i < num_j ? J[src[i]] : h[src[i]];
}

cudaError_t scatter_weights(double *arena, const int64_t *dst, const int32_t *src, int64_t num_j,
                            int64_t total, const double *J, const double *h,
                            cudaStream_t stream) {
    if (total <= 0) return cudaSuccess;
    const int64_t blocks = std::min<int64_t>((total + 255) / 256, 148 * 8);
    scatter_weights_kernel<<<(int)blocks, 256, 0, stream>>>(arena, dst, src, num_j, total, J, h);
    return cudaGetLastError();
}

cudaError_t upload_jump_table(const uint32_t table[][4], cudaStream_t stream) {
    return cudaMemcpyToSymbolAsync(g_jump_nib, table, sizeof(uint4) * kJumpTable, 0,
                                   cudaMemcpyHostToDevice, stream);
}

cudaError_t launch_sa(int variant, const LaunchArgs &args, int grid, int warps_per_cta,
                      int region_bytes, cudaStream_t stream) {
    const KernelFn k = kernel_for(variant);
    if (!k) return cudaErrorInvalidValue;
    const size_t smem = (size_t)warps_per_cta * (size_t)region_bytes;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k<<<grid, warps_per_cta * 32, smem, stream>>>(args, warps_per_cta, region_bytes);
    return cudaGetLastError();
}

cudaError_t kernel_occupancy(int variant, int warps_per_cta, int region_bytes, int *ctas_per_sm) {
    const KernelFn k = kernel_for(variant);
    if (!k) return cudaErrorInvalidValue;
    const size_t smem = (size_t)warps_per_cta * (size_t)region_bytes;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas_per_sm, k, warps_per_cta * 32, smem);
}

using SdKernel = void (*)(SdArgs, int, int);

static SdKernel sd_kernel_for(bool sparse, bool smem) {
    if (sparse) return smem ? sd_warp_kernel<true, true> : sd_warp_kernel<true, false>;
    return smem ? sd_warp_kernel<false, true> : sd_warp_kernel<false, false>;
}

cudaError_t launch_sd(bool sparse, bool smem, const SdArgs &args, int grid, int warps_per_cta,
                      int region_bytes, cudaStream_t stream) {
    const SdKernel k = sd_kernel_for(sparse, smem);
    const size_t bytes = (size_t)warps_per_cta * (size_t)region_bytes;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) return e;
    k<<<grid, warps_per_cta * 32, bytes, stream>>>(args, warps_per_cta, region_bytes);
    return cudaGetLastError();
}

cudaError_t sd_occupancy(bool sparse, bool smem, int warps_per_cta, int region_bytes,
                         int *ctas_per_sm) {
    const SdKernel k = sd_kernel_for(sparse, smem);
    const size_t bytes = (size_t)warps_per_cta * (size_t)region_bytes;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas_per_sm, k, warps_per_cta * 32, bytes);
}

using RmcKernel = void (*)(RmcArgs);

cudaError_t launch_rmc(bool random_order, int proposal, const RmcArgs &args, int grid,
                       int block, cudaStream_t stream) {
    static const RmcKernel table[2][4] = {
        {rmc_kernel<false, 0>, rmc_kernel<false, 1>, rmc_kernel<false, 2>, rmc_kernel<false, 3>},
        {rmc_kernel<true, 0>, rmc_kernel<true, 1>, rmc_kernel<true, 2>, rmc_kernel<true, 3>}};
    if (proposal < 0 || proposal > 3) return cudaErrorInvalidValue;
    table[random_order ? 1 : 0][proposal]<<<grid, block, 0, stream>>>(args);
    return cudaGetLastError();
}

cudaError_t launch_pimc(bool chain_update, const PimcArgs &args, int grid, int block,
                        cudaStream_t stream) {
    if (chain_update)
        pimc_kernel<true><<<grid, block, 0, stream>>>(args);
    else
        pimc_kernel<false><<<grid, block, 0, stream>>>(args);
    return cudaGetLastError();
}

}  // namespace b200sa
