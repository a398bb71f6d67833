// C ABI entry of the path-integral Monte Carlo annealing (b200sa_path_anneal):
// the host side of the drop-in for the reference's SQA general_simulated_annealing
// (dwave/samplers/sqa/src/localPIMC.cpp:585-715, bound at
// dwave/samplers/sqa/pimc_annealing.pyx:45-283).  The kernel and the
// arithmetic it follows are in pimc_kernel.cuh.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "pack.h"
#include "plan.h"

using namespace b200sa;
using namespace b200sa::host;

namespace {

// Break capacity when the caller gives none: proposals per update are about
// Poisson(Gamma); the bound sits more than ten standard deviations above the
// largest Gamma of the schedule.
int auto_capacity(const double *hd, int num_betas) {
    double g = 0.0;
    for (int b = 0; b < num_betas; ++b)
        if (std::isfinite(hd[b])) g = std::max(g, std::fabs(hd[b]));
    const double cap = g + 10.0 * std::sqrt(g) + 16.0;
    return (int)std::min(1e6, std::ceil(cap / 4.0) * 4.0);
}

}  // namespace

extern "C" int b200sa_path_anneal(
    int32_t num_vars, const double *h, int64_t num_couplers, const int32_t *coupler_starts,
    const int32_t *coupler_ends, const double *coupler_weights, int32_t num_samples,
    int8_t *states, double *energies, int32_t sweeps_per_beta, int32_t num_betas,
    const double *hp_field, const double *hd_field, double chain_coupler_strength,
    int32_t qubits_per_chain, int32_t qubits_per_update, const uint32_t *seeds,
    int32_t num_seeds, int32_t project_inputs, int32_t project_outputs, int32_t *num_breaks,
    const int32_t *breaks_in, int64_t breaks_in_size, int32_t *breaks_out,
    int64_t breaks_out_size, int8_t *statistics, int32_t schedule_sample_interval,
    int32_t break_capacity, int32_t device, int64_t *near_ties, char *err, size_t errlen) {
    if (near_ties) *near_ties = 0;
    if (num_samples < 0 || num_vars < 0 || num_couplers < 0 || sweeps_per_beta < 0 ||
        num_betas < 0 || schedule_sample_interval < 0 || break_capacity < 0 ||
        breaks_in_size < 0 || breaks_out_size < 0)
        return set_err(err, errlen, B200SA_EINVAL, "negative size");
    if (num_samples == 0 || num_vars == 0) {  // pimc_annealing.pyx:185-191
        if (num_samples > 0 && !energies)
            return set_err(err, errlen, B200SA_EINVAL, "energies is NULL");
        for (int32_t r = 0; r < num_samples; ++r) energies[r] = 0.0;
        return num_samples;
    }
    if (!states || !energies || !h || (num_betas > 0 && (!hp_field || !hd_field)))
        return set_err(err, errlen, B200SA_EINVAL, "null input or output array");
    if (num_couplers > 0 && (!coupler_starts || !coupler_ends || !coupler_weights))
        return set_err(err, errlen, B200SA_EINVAL, "coupler arrays are NULL");
    if (!seeds || (num_seeds != 1 && num_seeds != num_samples))
        return set_err(err, errlen, B200SA_EINVAL,
                       "num_seeds must be 1 (one continued stream) or num_samples (per sample)");
    if (qubits_per_chain < 1)
        return set_err(err, errlen, B200SA_EINVAL, "qubits_per_chain must be at least 1");
    const bool chain = qubits_per_update != 1;
    const int chains = num_vars / qubits_per_chain;
    if (chain && chains < 1)
        return set_err(err, errlen, B200SA_EINVAL,
                       "qubits_per_chain exceeds the number of variables");
    if ((!project_inputs || !project_outputs) && !num_breaks)
        return set_err(err, errlen, B200SA_EINVAL, "num_breaks is NULL");
    if (!project_outputs && breaks_out_size > 0 && !breaks_out)
        return set_err(err, errlen, B200SA_EINVAL, "breaks_out is NULL");
    if (schedule_sample_interval && !statistics)
        return set_err(err, errlen, B200SA_EINVAL, "statistics is NULL");
    for (int64_t c = 0; c < num_couplers; ++c) {  // localPIMC.cpp:644-646
        const int32_t a = coupler_starts[c], b = coupler_ends[c];
        if (a < 0 || b < 0 || a >= num_vars || b >= num_vars)
            return set_err(err, errlen, B200SA_EINVAL,
                           "coupler indexes contain an invalid variable");
    }
    const size_t n = (size_t)num_vars, R = (size_t)num_samples, m = (size_t)num_couplers;
    // Quantum initial states: num_breaks[r][v] positions per variable, in order.
    int max_in = 0;
    if (!project_inputs) {
        int64_t total = 0;
        for (size_t i = 0; i < R * n; ++i) {
            if (num_breaks[i] < 0)
                return set_err(err, errlen, B200SA_EINVAL, "negative entry in num_breaks");
            total += num_breaks[i];
            max_in = std::max(max_in, num_breaks[i]);
        }
        if (total > breaks_in_size || (total > 0 && !breaks_in))
            return set_err(err, errlen, B200SA_EINVAL,
                           "breaks_in holds fewer positions than num_breaks asks for");
    }
    const int cap_props = break_capacity ? break_capacity : auto_capacity(hd_field, num_betas);
    const int cap_breaks = std::max(cap_props, (max_in + 3) & ~3);
    const int Q = chain ? qubits_per_chain : 1;
    const int64_t C = (int64_t)cap_props + cap_breaks;
    // props, itf [Q][C], sv [Q * C], off [Q + 1], lab [Q * C], parent [Q * C], pair [2C]
    const int64_t scratch_ints = cap_props + 4 * Q * C + Q + 1 + 2 * C;
    const int64_t scratch_doubles = Q * C;
    const bool shared = num_seeds == 1 && num_samples > 1;
    const size_t slots = shared ? 1 : R;
    // Seed 0 asks the reference for a nondeterministic generator
    // (localPIMC.cpp:578-587); here it draws a nonzero seed from the device.
    std::vector<uint32_t> hseeds(seeds, seeds + num_seeds);
    for (auto &s : hseeds) {
        if (s == 0) {
            std::random_device rd;
            do s = rd(); while (s == 0);
        }
    }
    // Schedule indices divisible by the interval; none for an empty schedule
    // (the bindings' floor division gives 0 there too).
    const int points = schedule_sample_interval && num_betas > 0
                           ? 1 + (num_betas - 1) / schedule_sample_interval
                           : 0;

    b200sa_problem q{};
    q.num_vars = num_vars;
    q.num_couplers = num_couplers;
    q.coupler_starts = coupler_starts;
    q.coupler_ends = coupler_ends;
    q.coupler_weights = coupler_weights;
    PackedAdjacency adj;  // coupler input order (localPIMC.cpp:633-655)
    pack_adjacency(q, adj);
    std::vector<uint2> vinfo(n);
    for (size_t v = 0; v < n; ++v)
        vinfo[v] = make_uint2(adj.vinfo[2 * v], adj.vinfo[2 * v + 1] & kDegMask);

    DeviceGuard guard;
    cudaDeviceProp prop;
    int rc = select_device(device, prop, err, errlen);
    if (rc) return rc;
    DevArray<uint2> dvinfo;
    DevArray<int32_t> dcol, dcu, dcv, dcnt, dbrk, dscr_i, dflag;
    DevArray<double> dw, dh, dcw, dhp, dhd, den, dscr_d;
    DevArray<uint32_t> dseeds, dmt;
    DevArray<int8_t> dst, dstats;
    DevArray<unsigned long long> dnear;
    const size_t list_words = R * n * (size_t)cap_breaks;
    B200SA_CUDA(dvinfo.alloc(n));
    B200SA_CUDA(dcol.alloc(std::max<size_t>(2 * m, 1)));
    B200SA_CUDA(dw.alloc(std::max<size_t>(2 * m, 1)));
    B200SA_CUDA(dcu.alloc(std::max<size_t>(m, 1)));
    B200SA_CUDA(dcv.alloc(std::max<size_t>(m, 1)));
    B200SA_CUDA(dcw.alloc(std::max<size_t>(m, 1)));
    B200SA_CUDA(dh.alloc(n));
    B200SA_CUDA(dhp.alloc(std::max<size_t>((size_t)num_betas, 1)));
    B200SA_CUDA(dhd.alloc(std::max<size_t>((size_t)num_betas, 1)));
    B200SA_CUDA(dseeds.alloc((size_t)num_seeds));
    B200SA_CUDA(dst.alloc(n * R));
    B200SA_CUDA(dcnt.alloc(n * R));
    B200SA_CUDA(dbrk.alloc(list_words));
    B200SA_CUDA(dmt.alloc(slots * kMtWords));
    B200SA_CUDA(dscr_i.alloc(slots * (size_t)scratch_ints));
    B200SA_CUDA(dscr_d.alloc(slots * (size_t)scratch_doubles));
    B200SA_CUDA(den.alloc(R));
    B200SA_CUDA(dnear.alloc(1));
    B200SA_CUDA(dflag.alloc(1));
    if (points) B200SA_CUDA(dstats.alloc(R * (size_t)points * n));
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
    B200SA_CUDA(up(dhp.ptr, hp_field, 8 * (size_t)num_betas));
    B200SA_CUDA(up(dhd.ptr, hd_field, 8 * (size_t)num_betas));
    B200SA_CUDA(up(dseeds.ptr, hseeds.data(), 4 * (size_t)num_seeds));
    B200SA_CUDA(up(dst.ptr, states, n * R));
    if (project_inputs) {
        B200SA_CUDA(cudaMemset(dcnt.ptr, 0, 4 * n * R));
    } else {
        std::vector<int32_t> lists(list_words, 0);
        size_t pos = 0;
        for (size_t i = 0; i < R * n; ++i)
            for (int k = 0; k < num_breaks[i]; ++k)
                lists[i * (size_t)cap_breaks + k] = breaks_in[pos++];
        B200SA_CUDA(up(dcnt.ptr, num_breaks, 4 * n * R));
        B200SA_CUDA(up(dbrk.ptr, lists.data(), 4 * list_words));
    }
    B200SA_CUDA(cudaMemset(dnear.ptr, 0, sizeof(unsigned long long)));
    B200SA_CUDA(cudaMemset(dflag.ptr, 0, sizeof(int32_t)));
    PimcArgs a{};
    a.n = num_vars;
    a.m = num_couplers;
    a.vinfo = dvinfo.ptr;
    a.col = dcol.ptr;
    a.w = dw.ptr;
    a.h = dh.ptr;
    a.cu = dcu.ptr;
    a.cv = dcv.ptr;
    a.cw = dcw.ptr;
    a.hp = dhp.ptr;
    a.hd = dhd.ptr;
    a.num_betas = num_betas;
    a.sweeps_per_beta = sweeps_per_beta;
    a.jchain = chain_coupler_strength;
    a.qpc = qubits_per_chain;
    a.chains = chains;
    a.seeds = dseeds.ptr;
    a.shared_stream = shared ? 1 : 0;
    a.num_samples = num_samples;
    a.states = dst.ptr;
    a.counts = dcnt.ptr;
    a.breaks = dbrk.ptr;
    a.cap_breaks = cap_breaks;
    a.cap_props = cap_props;
    a.mt = dmt.ptr;
    a.scratch_i = dscr_i.ptr;
    a.scratch_d = dscr_d.ptr;
    a.scratch_ints = scratch_ints;
    a.scratch_doubles = scratch_doubles;
    a.energies = den.ptr;
    a.stats = points ? dstats.ptr : nullptr;
    a.interval = schedule_sample_interval;
    a.near = dnear.ptr;
    a.overflow = dflag.ptr;
    // One latency-bound chain per sample: small CTAs spread the samples over
    // every SM.
    const int sms = prop.multiProcessorCount;
    const int block = R >= (size_t)sms * 32 * 64 ? 64 : 32;
    const int grid = shared ? 1 : (int)((R + block - 1) / block);
    B200SA_CUDA(launch_pimc(chain, a, grid, block, nullptr));
    B200SA_CUDA(cudaDeviceSynchronize());
    int32_t overflow = 0;
    B200SA_CUDA(cudaMemcpy(&overflow, dflag.ptr, sizeof(overflow), cudaMemcpyDeviceToHost));
    if (overflow)
        return set_err(err, errlen, B200SA_ERANGE,
                       "a break list or the break proposals of one update exceeded the capacity " +
                           std::to_string(cap_props) +
                           "; call again with a larger break_capacity");
    B200SA_CUDA(cudaMemcpy(states, dst.ptr, n * R, cudaMemcpyDeviceToHost));
    B200SA_CUDA(cudaMemcpy(energies, den.ptr, 8 * R, cudaMemcpyDeviceToHost));
    unsigned long long near = 0;
    B200SA_CUDA(cudaMemcpy(&near, dnear.ptr, sizeof(near), cudaMemcpyDeviceToHost));
    if (near_ties) *near_ties = (int64_t)near;
    if (points)
        B200SA_CUDA(cudaMemcpy(statistics, dstats.ptr, R * (size_t)points * n,
                               cudaMemcpyDeviceToHost));
    if (!project_outputs) {
        // readBreaks (localPIMC.cpp:185-200) sample after sample: a variable's
        // breaks are written only while the rest of the buffer holds them all,
        // and every sample's start moves on by its total count.
        std::vector<int32_t> lists(list_words);
        B200SA_CUDA(cudaMemcpy(num_breaks, dcnt.ptr, 4 * n * R, cudaMemcpyDeviceToHost));
        B200SA_CUDA(cudaMemcpy(lists.data(), dbrk.ptr, 4 * list_words, cudaMemcpyDeviceToHost));
        int64_t start = 0;
        for (size_t r = 0; r < R; ++r) {
            int64_t capacity = breaks_out_size - start;
            int64_t p = start, total = 0;
            for (size_t v = 0; v < n; ++v) {
                const int c = num_breaks[r * n + v];
                if (capacity >= c) {
                    if (c) std::memcpy(breaks_out + p, &lists[(r * n + v) * (size_t)cap_breaks],
                                       sizeof(int32_t) * (size_t)c);
                    p += c;
                    capacity -= c;
                }
                total += c;
            }
            start += total;
        }
    }
    return num_samples;
}
