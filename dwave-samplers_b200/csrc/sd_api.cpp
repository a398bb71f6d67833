// C ABI entry of the steepest descent (b200sa_steepest_descent): the host
// side of the drop-in for the reference's steepest_gradient_descent
// (dwave/samplers/greedy/src/descent.cpp:315-405).  The kernel and the
// arithmetic it follows are in sd_kernel.cuh.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "plan.h"

using namespace b200sa;
using namespace b200sa::host;

extern "C" int b200sa_steepest_descent(int32_t num_vars, const double *h, int64_t num_couplers,
                                       const int32_t *coupler_starts,
                                       const int32_t *coupler_ends,
                                       const double *coupler_weights, int32_t num_samples,
                                       int8_t *states, double *energies, uint32_t *num_steps,
                                       int32_t large_sparse_opt, uint32_t max_steps,
                                       int32_t device, char *err, size_t errlen) {
    if (num_samples < 0) return set_err(err, errlen, B200SA_EINVAL, "num_samples < 0");
    if (num_samples == 0) return 0;
    if ((!states && num_vars > 0) || !energies || !num_steps)
        return set_err(err, errlen, B200SA_EINVAL, "states, energies or num_steps is NULL");
    if (num_vars == 0) {  // descent.cpp:124-127: no variables, no steps, energy 0
        for (int32_t r = 0; r < num_samples; ++r) {
            energies[r] = 0.0;
            num_steps[r] = 0;
        }
        return num_samples;
    }
    if (max_steps == 0)
        max_steps = (uint32_t)std::min<int64_t>(UINT32_MAX, 1000 * (int64_t)num_vars + 1000000);
    // The plan packs the problem (order-preserving adjacency, COO for the
    // energy) exactly as for annealing; its schedule is empty.
    std::vector<uint64_t> seeds((size_t)num_samples, 1);
    b200sa_problem q{};
    q.num_vars = num_vars;
    q.h = h;
    q.num_couplers = num_couplers;
    q.coupler_starts = coupler_starts;
    q.coupler_ends = coupler_ends;
    q.coupler_weights = coupler_weights;
    q.num_reads = num_samples;
    q.seeds = seeds.data();
    q.varorder = B200SA_SEQUENTIAL;
    q.proposal = B200SA_METROPOLIS;
    b200sa_plan plan = nullptr;
    int rc = b200sa_plan_create(&q, 1, device, &plan, err, errlen);
    if (rc) return rc;
    std::unique_ptr<b200sa_plan_s, int (*)(b200sa_plan)> hold(plan, b200sa_plan_destroy);
    DeviceGuard guard;
    B200SA_CUDA(cudaSetDevice(plan->device));
    const bool sparse = large_sparse_opt != 0;
    const int smem_blk = (int)plan->prop.sharedMemPerBlockOptin;
    const int sms = plan->prop.multiProcessorCount;
    // Shared-memory state when three warps' regions fit on an SM.
    const bool onchip = 3 * sd_region_bytes(num_vars) + 3 * 1024 <=
                        (int)plan->prop.sharedMemPerMultiprocessor;
    const int cap = onchip ? num_vars : 0;
    const int region = sd_region_bytes(cap);
    int best_w = 1, best = 0;
    for (int w = 1; w <= kMaxThreadsPerCta / 32 && w * region <= smem_blk; ++w) {
        int ctas = 0;
        B200SA_CUDA(sd_occupancy(sparse, onchip, w, region, &ctas));
        if (ctas * w > best) {
            best = ctas * w;
            best_w = w;
        }
    }
    if (best == 0) return set_err(err, errlen, B200SA_ECUDA, "descent kernel does not fit");
    const int w = (int)std::min<int64_t>(best_w, std::max<int64_t>(1, (num_samples + sms - 1) / sms));
    int ctas = 0;
    B200SA_CUDA(sd_occupancy(sparse, onchip, w, region, &ctas));
    const int grid = (int)std::max<int64_t>(
        1, std::min<int64_t>((int64_t)sms * std::max(ctas, 1), (num_samples + w - 1) / w));
    const int64_t slots = (int64_t)grid * w;
    const int64_t stride = ((int64_t)num_vars + 15) & ~int64_t(15);
    DevArray<int8_t> dstates;
    DevArray<double> den, sfe;
    DevArray<int8_t> ss;
    DevArray<uint32_t> dsteps;
    DevArray<unsigned long long> counters;  // queue head, capped samples
    const size_t total = (size_t)num_samples * (size_t)num_vars;
    B200SA_CUDA(dstates.alloc(total));
    B200SA_CUDA(den.alloc((size_t)num_samples));
    B200SA_CUDA(dsteps.alloc((size_t)num_samples));
    B200SA_CUDA(counters.alloc(2));
    if (!onchip) {
        B200SA_CUDA(sfe.alloc((size_t)(slots * stride)));
        B200SA_CUDA(ss.alloc((size_t)(slots * stride)));
    }
    cudaStream_t st = plan->stream;
    B200SA_CUDA(cudaMemcpyAsync(dstates.ptr, states, total, cudaMemcpyHostToDevice, st));
    B200SA_CUDA(cudaMemsetAsync(counters.ptr, 0, 2 * sizeof(unsigned long long), st));
    SdArgs a{};
    a.problem = plan->dprobs.ptr;
    a.items = plan->items_plain.ptr;
    a.num_items = num_samples;
    a.queue_head = counters.ptr;
    a.states_in = dstates.ptr;
    a.states_out = dstates.ptr;
    a.energies = den.ptr;
    a.steps = dsteps.ptr;
    a.max_steps = max_steps;
    a.smem_cap_n = cap;
    a.scratch_fe = sfe.ptr;
    a.scratch_s = ss.ptr;
    a.scratch_stride = stride;
    a.capped = counters.ptr + 1;
    B200SA_CUDA(launch_sd(sparse, onchip, a, grid, w, region, st));
    unsigned long long capped = 0;
    B200SA_CUDA(cudaMemcpyAsync(states, dstates.ptr, total, cudaMemcpyDeviceToHost, st));
    B200SA_CUDA(cudaMemcpyAsync(energies, den.ptr, sizeof(double) * (size_t)num_samples,
                                cudaMemcpyDeviceToHost, st));
    B200SA_CUDA(cudaMemcpyAsync(num_steps, dsteps.ptr, sizeof(uint32_t) * (size_t)num_samples,
                                cudaMemcpyDeviceToHost, st));
    B200SA_CUDA(cudaMemcpyAsync(&capped, counters.ptr + 1, sizeof(capped),
                                cudaMemcpyDeviceToHost, st));
    B200SA_CUDA(cudaStreamSynchronize(st));
    if (capped)
        return set_err(err, errlen, B200SA_ETIMEOUT,
                       std::to_string(capped) + " sample(s) stopped after max_steps = " +
                           std::to_string(max_steps) +
                           " steps without reaching a minimum (a positive self-loop, or spins "
                           "other than +-1, can make descent cycle)");
    return num_samples;
}
