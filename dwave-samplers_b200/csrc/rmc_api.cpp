// C ABI entry of the rotor-model annealing (b200sa_rotor_anneal): the host
// side of the drop-in for the reference's SQA rotor Monte Carlo
// general_simulated_annealing (dwave/samplers/sqa/src/cpu_rotormc.cpp:368-563,
// bound at dwave/samplers/sqa/rotormc_annealing.pyx:54-236).  The kernel and
// the arithmetic it follows are in rmc_kernel.cuh.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "pack.h"
#include "plan.h"

using namespace b200sa;
using namespace b200sa::host;

extern "C" int b200sa_rotor_anneal(int32_t num_vars, const double *h, int64_t num_couplers,
                                   const int32_t *coupler_starts, const int32_t *coupler_ends,
                                   const double *coupler_weights, const double *trans_fields,
                                   int32_t num_samples, uint8_t *states, double *energies,
                                   int32_t sweeps_per_beta, int32_t num_betas,
                                   const double *hp_field, const double *hd_field,
                                   const uint64_t *seeds, int32_t num_seeds,
                                   int32_t randomize_order, int32_t proposal,
                                   uint8_t *statistics, int32_t schedule_sample_interval,
                                   int32_t device, int64_t *near_ties, char *err,
                                   size_t errlen) {
    if (near_ties) *near_ties = 0;
    if (num_samples < 0 || num_vars < 0 || num_couplers < 0 || sweeps_per_beta < 0 ||
        num_betas < 0 || schedule_sample_interval < 0)
        return set_err(err, errlen, B200SA_EINVAL, "negative size");
    if (proposal < 0 || proposal > 3)
        return set_err(err, errlen, B200SA_EINVAL,
                       "proposal must be 0 (GibbsNonErgodic), 1 (MetropolisNonErgodic), "
                       "2 (MetropolisUniform) or 3 (MetropolisTF)");
    if (num_samples == 0 || num_vars == 0) {  // rotormc_annealing.pyx:161-164
        if (num_samples > 0 && !energies)
            return set_err(err, errlen, B200SA_EINVAL, "energies is NULL");
        for (int32_t r = 0; r < num_samples; ++r) energies[r] = 0.0;
        return num_samples;
    }
    if (!states || !energies || !h || !trans_fields || (num_betas > 0 && (!hp_field || !hd_field)))
        return set_err(err, errlen, B200SA_EINVAL, "null input or output array");
    if (num_couplers > 0 && (!coupler_starts || !coupler_ends || !coupler_weights))
        return set_err(err, errlen, B200SA_EINVAL, "coupler arrays are NULL");
    if (!seeds || (num_seeds != 1 && num_seeds != num_samples))
        return set_err(err, errlen, B200SA_EINVAL,
                       "num_seeds must be 1 (one continued stream) or num_samples (per sample)");
    for (int64_t c = 0; c < num_couplers; ++c) {  // cpu_rotormc.cpp:411-413
        const int32_t a = coupler_starts[c], b = coupler_ends[c];
        if (a < 0 || b < 0 || a >= num_vars || b >= num_vars)
            return set_err(err, errlen, B200SA_EINVAL,
                           "coupler indexes contain an invalid variable");
    }
    // Adjacency in coupler input order (cpu_rotormc.cpp:399-424).
    b200sa_problem q{};
    q.num_vars = num_vars;
    q.num_couplers = num_couplers;
    q.coupler_starts = coupler_starts;
    q.coupler_ends = coupler_ends;
    q.coupler_weights = coupler_weights;
    PackedAdjacency adj;
    pack_adjacency(q, adj);
    // cos and |sin| of the 256 angles, as cpu_rotormc.cpp:377-383.
    double cos_t[256], sin_t[256];
    for (int i = 0; i < 256; ++i) {
        cos_t[i] = std::cos(2 * i * M_PI / 256);
        sin_t[i] = std::abs(std::sin(2 * i * M_PI / 256));
    }
    DeviceGuard guard;
    cudaDeviceProp prop;
    int rc = select_device(device, prop, err, errlen);
    if (rc) return rc;
    const bool shared = num_seeds == 1 && num_samples > 1;
    // Schedule indices divisible by the interval; none for an empty schedule
    // (the bindings' floor division gives 0 there too).
    const int points = schedule_sample_interval && num_betas > 0
                           ? 1 + (num_betas - 1) / schedule_sample_interval
                           : 0;
    const size_t n = (size_t)num_vars, R = (size_t)num_samples, m = (size_t)num_couplers;
    DevArray<uint2> dvinfo;
    DevArray<int32_t> dcol, dcu, dcv;
    DevArray<double> dw, dh, dtf, dcw, dhp, dhd, dde, den, dtab;
    DevArray<uint64_t> dseeds;
    DevArray<uint8_t> dst, drows, dstats;
    DevArray<unsigned long long> dnear;
    std::vector<uint2> vinfo(n);
    for (size_t v = 0; v < n; ++v)
        vinfo[v] = make_uint2(adj.vinfo[2 * v], adj.vinfo[2 * v + 1] & kDegMask);
    std::vector<double> tab(512);
    std::copy(cos_t, cos_t + 256, tab.begin());
    std::copy(sin_t, sin_t + 256, tab.begin() + 256);
    B200SA_CUDA(dvinfo.alloc(n));
    B200SA_CUDA(dcol.alloc(std::max<size_t>(2 * m, 1)));
    B200SA_CUDA(dw.alloc(std::max<size_t>(2 * m, 1)));
    B200SA_CUDA(dcu.alloc(std::max<size_t>(m, 1)));
    B200SA_CUDA(dcv.alloc(std::max<size_t>(m, 1)));
    B200SA_CUDA(dcw.alloc(std::max<size_t>(m, 1)));
    B200SA_CUDA(dh.alloc(n));
    B200SA_CUDA(dtf.alloc(n));
    B200SA_CUDA(dhp.alloc(std::max<size_t>((size_t)num_betas, 1)));
    B200SA_CUDA(dhd.alloc(std::max<size_t>((size_t)num_betas, 1)));
    B200SA_CUDA(dtab.alloc(512));
    B200SA_CUDA(dseeds.alloc((size_t)num_seeds));
    B200SA_CUDA(dst.alloc(n * R));
    B200SA_CUDA(drows.alloc(n * R));
    B200SA_CUDA(dde.alloc(n * R));
    B200SA_CUDA(den.alloc(R));
    B200SA_CUDA(dnear.alloc(1));
    if (statistics && points) B200SA_CUDA(dstats.alloc(R * (size_t)points * n));
    auto up = [](void *dst_, const void *src, size_t bytes) {
        return bytes ? cudaMemcpy(dst_, src, bytes, cudaMemcpyHostToDevice) : cudaSuccess;
    };
    B200SA_CUDA(up(dvinfo.ptr, vinfo.data(), sizeof(uint2) * n));
    B200SA_CUDA(up(dcol.ptr, adj.col.data(), 4 * 2 * m));
    B200SA_CUDA(up(dw.ptr, adj.w.data(), 8 * 2 * m));
    B200SA_CUDA(up(dcu.ptr, coupler_starts, 4 * m));
    B200SA_CUDA(up(dcv.ptr, coupler_ends, 4 * m));
    B200SA_CUDA(up(dcw.ptr, coupler_weights, 8 * m));
    B200SA_CUDA(up(dh.ptr, h, 8 * n));
    B200SA_CUDA(up(dtf.ptr, trans_fields, 8 * n));
    B200SA_CUDA(up(dhp.ptr, hp_field, 8 * (size_t)num_betas));
    B200SA_CUDA(up(dhd.ptr, hd_field, 8 * (size_t)num_betas));
    B200SA_CUDA(up(dtab.ptr, tab.data(), 8 * 512));
    B200SA_CUDA(up(dseeds.ptr, seeds, 8 * (size_t)num_seeds));
    B200SA_CUDA(up(drows.ptr, states, n * R));
    B200SA_CUDA(cudaMemset(dnear.ptr, 0, sizeof(unsigned long long)));
    RmcArgs a{};
    a.n = num_vars;
    a.m = num_couplers;
    a.vinfo = dvinfo.ptr;
    a.col = dcol.ptr;
    a.w = dw.ptr;
    a.h = dh.ptr;
    a.tf = dtf.ptr;
    a.cu = dcu.ptr;
    a.cv = dcv.ptr;
    a.cw = dcw.ptr;
    a.hp = dhp.ptr;
    a.hd = dhd.ptr;
    a.num_betas = num_betas;
    a.sweeps_per_beta = sweeps_per_beta;
    a.seeds = dseeds.ptr;
    a.shared_stream = shared ? 1 : 0;
    a.num_samples = num_samples;
    a.rows = drows.ptr;
    a.states = dst.ptr;
    a.de = dde.ptr;
    a.energies = den.ptr;
    a.stats = (statistics && points) ? dstats.ptr : nullptr;
    a.interval = schedule_sample_interval;
    a.cos_table = dtab.ptr;
    a.sin_table = dtab.ptr + 256;
    a.near = dnear.ptr;
    // Each read is one latency-bound chain: small CTAs spread the reads over
    // every SM (up to 32 CTAs per SM); 64-thread CTAs once the reads fill them.
    const int sms = prop.multiProcessorCount;
    const int block = R >= (size_t)sms * 32 * 64 ? 64 : 32;
    const int grid = shared ? 1 : (int)((R + block - 1) / block);
    B200SA_CUDA(launch_rmc(randomize_order != 0, proposal, a, grid, block, nullptr));
    B200SA_CUDA(cudaDeviceSynchronize());
    B200SA_CUDA(cudaMemcpy(states, drows.ptr, n * R, cudaMemcpyDeviceToHost));
    B200SA_CUDA(cudaMemcpy(energies, den.ptr, 8 * R, cudaMemcpyDeviceToHost));
    unsigned long long near = 0;
    B200SA_CUDA(cudaMemcpy(&near, dnear.ptr, sizeof(near), cudaMemcpyDeviceToHost));
    if (near_ties) *near_ties = (int64_t)near;
    if (statistics && points) {
        std::vector<uint8_t> blocks(R * (size_t)points * n);
        B200SA_CUDA(cudaMemcpy(blocks.data(), dstats.ptr, blocks.size(), cudaMemcpyDeviceToHost));
        // One continued stream is one reference call: sample r's block starts
        // at r * n * (num_betas / interval) (cpu_rotormc.cpp:445) and later
        // samples overwrite any overlap.  Per-sample seeds are one call per
        // sample: blocks side by side.
        const size_t stride = shared ? n * (size_t)(num_betas / schedule_sample_interval)
                                     : (size_t)points * n;
        for (size_t r = 0; r < R; ++r)
            std::memcpy(statistics + r * stride, blocks.data() + r * (size_t)points * n,
                        (size_t)points * n);
    }
    return num_samples;
}
