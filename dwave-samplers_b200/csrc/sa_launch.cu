// Kernel entry point: warps take (problem, read) work items, either from a
// device work-queue head (persistent mode: one launch for a whole batch) or
// by a static stride (plain mode: one launch per problem).
#include <cuda_runtime.h>

#include "sa_kernel.cuh"
#include "sa_launch.h"

namespace b200sa {

__global__ void __launch_bounds__(kMaxThreadsPerCta, 1)
    sa_warp_kernel(LaunchArgs A, int warps_per_cta, int region_bytes) {
    extern __shared__ __align__(16) uint8_t smem[];
    const unsigned lane = threadIdx.x & 31u;
    const int wid = (int)(threadIdx.x >> 5);
    uint8_t *region = smem + (size_t)wid * (size_t)region_bytes;
    uint64_t *ring = reinterpret_cast<uint64_t *>(region);
    double *de_s = reinterpret_cast<double *>(region + kRing * sizeof(uint64_t));
    int8_t *sp_s = reinterpret_cast<int8_t *>(region + kRing * sizeof(uint64_t) +
                                              (size_t)A.smem_cap_n * sizeof(double));
    const int64_t gw = (int64_t)blockIdx.x * warps_per_cta + wid;
    const int64_t total_warps = (int64_t)gridDim.x * warps_per_cta;
    if (A.shared_stream && gw != 0) return;

    RingState rs;
    bool stream_live = false;
    if (A.shared_stream && A.carry_in) {
        for (int i = lane; i < kRing; i += 32) ring[i] = A.rng_carry[i];
        rs.t0 = A.rng_carry[kRing + 2 * lane];
        rs.t1 = A.rng_carry[kRing + 2 * lane + 1];
        rs.q = A.rng_carry[kRing + kCarryLaneWords];
        rs.base = A.rng_carry[kRing + kCarryLaneWords + 1];
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
        const ProblemDev &P = A.problems[pi];
        const int64_t rd = P.read_offset + r;
        if (!stream_live) {
            ring_init(ring, rs, A.seeds[rd], lane);
            stream_live = A.shared_stream != 0;
        }
        const int8_t *src = A.states_in + P.state_offset + (int64_t)r * P.n;
        int8_t *dst = A.states_out + P.state_offset + (int64_t)r * P.n;
        Counters cnt = {0ull, 0ull, 0u};
        if (P.n <= A.smem_cap_n) {
            anneal_dispatch<true>(P, src, dst, &A.energies[rd], de_s, sp_s, ring,
                                  rs, lane, cnt);
        } else {
            double *de_g = A.scratch_de + gw * A.scratch_stride;
            int8_t *sp_g = A.scratch_s + gw * A.scratch_stride;
            anneal_dispatch<false>(P, src, dst, &A.energies[rd], de_g, sp_g, ring,
                                   rs, lane, cnt);
        }
        if (lane == 0) {
            A.stats[rd].flips = cnt.flips;
            A.stats[rd].passes = cnt.passes;
            A.stats[rd].near_ties = cnt.near;
        }
        if (!A.queue_head) it += A.shared_stream ? 1 : total_warps;
    }

    if (A.shared_stream && stream_live) {
        __syncwarp();
        for (int i = lane; i < kRing; i += 32) A.rng_carry[i] = ring[i];
        A.rng_carry[kRing + 2 * lane] = rs.t0;
        A.rng_carry[kRing + 2 * lane + 1] = rs.t1;
        if (lane == 0) {
            A.rng_carry[kRing + kCarryLaneWords] = rs.q;
            A.rng_carry[kRing + kCarryLaneWords + 1] = rs.base;
        }
    }
}

cudaError_t upload_jump_columns(const uint32_t cols[128][4], cudaStream_t stream) {
    return cudaMemcpyToSymbolAsync(c_jump, cols, sizeof(uint4) * 128, 0,
                                   cudaMemcpyHostToDevice, stream);
}

cudaError_t launch_sa(const LaunchArgs &args, int grid, int warps_per_cta,
                      int region_bytes, cudaStream_t stream) {
    const size_t smem = (size_t)warps_per_cta * (size_t)region_bytes;
    cudaError_t e = cudaFuncSetAttribute(
        sa_warp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    sa_warp_kernel<<<grid, warps_per_cta * 32, smem, stream>>>(args, warps_per_cta,
                                                               region_bytes);
    return cudaGetLastError();
}

cudaError_t kernel_occupancy(int warps_per_cta, int region_bytes, int *ctas_per_sm) {
    const size_t smem = (size_t)warps_per_cta * (size_t)region_bytes;
    cudaError_t e = cudaFuncSetAttribute(
        sa_warp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas_per_sm, sa_warp_kernel,
                                                         warps_per_cta * 32, smem);
}

}  // namespace b200sa
