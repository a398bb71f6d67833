// C ABI of the B200 simulated-annealing sampler (declared in include/b200sa.h).
//
// Host side of the drop-in for general_simulated_annealing
// (dwave/samplers/sa/src/cpu_sa.cpp:253-362): validation, order-preserving
// packing, device residency, launch configuration, interrupt polling in read
// order, and error codes in place of the reference's thrown exceptions.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <utility>
#include <vector>

#include "b200sa.h"
#include "pack.h"
#include "sa_launch.h"
#include "sa_types.h"

#include "plan.h"

using namespace b200sa;
using namespace b200sa::host;

namespace b200sa {
namespace host {

int select_device(int device, cudaDeviceProp &prop, char *err, size_t errlen) {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return set_err(err, errlen, B200SA_ENODEV, "no CUDA device available");
    }
    if (device < 0 || device >= count)
        return set_err(err, errlen, B200SA_ENODEV,
                       "device index " + std::to_string(device) + " out of range");
    B200SA_CUDA(cudaSetDevice(device));
    B200SA_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10)
        return set_err(err, errlen, B200SA_ENODEV,
                       std::string("this library is built for sm_100a (B200); device is ") +
                           prop.name + " sm_" + std::to_string(prop.major * 10 + prop.minor));
    return B200SA_OK;
}


// In-window resolution of the sequential sweep is on unless the environment
// sets B200SA_RESOLVE=0 (results are identical either way; for A/B timing).
bool resolve_allowed() {
    static const bool on = [] {
        const char *e = std::getenv("B200SA_RESOLVE");
        return !(e && e[0] == '0');
    }();
    return on;
}

// Banded delta energies are on unless the environment sets B200SA_BAND=0
// (results are identical either way; for A/B timing).
bool band_allowed() {
    static const bool on = [] {
        const char *e = std::getenv("B200SA_BAND");
        return !(e && e[0] == '0');
    }();
    return on;
}

// Dense updates are on unless the environment sets B200SA_DENSE=0 (results
// are identical either way; for A/B timing).
bool dense_allowed() {
    static const bool on = [] {
        const char *e = std::getenv("B200SA_DENSE");
        return !(e && e[0] == '0');
    }();
    return on;
}

const uint32_t (*jump_table())[4] {
    static uint32_t table[kJumpTable][4];
    static std::once_flag once;
    std::call_once(once, [] {
        uint32_t cols[128][4];
        rng_jump_columns(kHalf, cols);
        rng_jump_nibbles(cols, table);
    });
    return table;
}

int occupancy(b200sa_plan_s *P, int variant, int w, int region, int *ctas, char *err,
              size_t errlen) {
    auto key = std::make_pair((variant << 24) + w, region);
    auto it = P->occ_cache.find(key);
    if (it != P->occ_cache.end()) {
        *ctas = it->second;
        return B200SA_OK;
    }
    B200SA_CUDA(kernel_occupancy(variant, w, region, ctas));
    P->occ_cache[key] = *ctas;
    return B200SA_OK;
}

// Every warp anneals one read at a time; its shared region holds the RNG
// ring, the conflict scratch and, by the state location, the read's delta
// energies and spins, its spins only, or neither (the rest lives in a global
// slot, L2-resident).  Untuned, state is in shared memory whenever it fits
// and warps per CTA maximize resident warps per SM.
int shape_for(b200sa_plan_s *P, int kind, int32_t max_n_here, int64_t items, bool persistent,
              LaunchShape &out, char *err, size_t errlen, const TuneChoice *choice,
              int band_w_here) {
    const int smem_blk = (int)P->prop.sharedMemPerBlockOptin;
    const int tb = touch_bytes_for((kind & kKindRandom) != 0, max_n_here);
    if (kind & kKindRandom) band_w_here = 0;  // the band follows a sequential window
    int stage = choice && choice->set ? choice->staging : kStageShared;
    if (stage == kStageBand &&
        (!band_w_here ||
         region_bytes_for_stage(kStageBand, max_n_here, band_w_here) + tb > smem_blk))
        stage = kStageSpins;
    // The most resident warps per SM a location allows (occupancy rule).
    auto most_warps = [&](int st, int region, int *most) {
        *most = 0;
        const int var = kernel_variant(kind, st, 0);
        for (int w = 1; w <= kMaxThreadsPerCta / 32 && (int64_t)w * region <= smem_blk; ++w) {
            int ctas = 0;
            int rc = occupancy(P, var, w, region, &ctas, err, errlen);
            if (rc) return rc;
            *most = std::max(*most, ctas * w);
        }
        return (int)B200SA_OK;
    };
    // Untuned register budget: 128 registers for state on chip or in the band,
    // the 80-register kernel (24 warps per SM) for global slots, whose delta
    // energies are updated by L2 reductions and gain from more reads in flight.
    bool untuned_global = false;
    if (!(choice && choice->set) && stage == kStageShared && max_n_here > P->onchip_fast &&
        max_n_here <= P->onchip_max &&
        region_bytes_for_stage(kStageSpins, max_n_here) + tb <= smem_blk) {
        // Untuned, on chip but with fewer than 24 warps' regions per SM: the
        // spins stay in shared memory, the delta energies go to the global
        // slot (measured faster from n ~ 1000 on).
        stage = kStageSpins;
        untuned_global = true;
    }
    if (stage == kStageShared && max_n_here > P->onchip_max) {
        untuned_global = true;
        stage = kStageGlobal;
        // Untuned, above the on-chip size, banded: the band location (spins
        // and the band of delta energies around the window on chip) when
        // every item still gets a resident warp that way.
        const int band_region = region_bytes_for_stage(kStageBand, max_n_here, band_w_here) + tb;
        if (!(choice && choice->set) && band_w_here && band_region <= smem_blk) {
            int most = 0;
            int rc = most_warps(kStageBand, band_region, &most);
            if (rc) return rc;
            if (most > 0 && items <= (int64_t)P->prop.multiProcessorCount * most)
                stage = kStageBand;
        }
        // Untuned, above the on-chip size: keep the spins in shared memory
        // (delta energies in the global slot) when every item still gets a
        // resident warp that way; the spin reads of the neighbour updates
        // then stay on chip.
        const int spins_region = region_bytes_for_stage(kStageSpins, max_n_here) + tb;
        if (stage == kStageGlobal && !(choice && choice->set) && spins_region <= smem_blk) {
            int most = 0;
            int rc = most_warps(kStageSpins, spins_region, &most);
            if (rc) return rc;
            if (most > 0 && items <= (int64_t)P->prop.multiProcessorCount * most)
                stage = kStageSpins;
        }
    }
    if (stage == kStageSpins && region_bytes_for_stage(kStageSpins, max_n_here) + tb > smem_blk)
        stage = kStageGlobal;
    const int cap = stage == kStageGlobal ? 0 : max_n_here;
    const int band_cap = stage == kStageBand ? band_w_here : 0;
    const int region = region_bytes_for_stage(stage, cap, band_cap) + tb;
    out.touch_bytes = tb;
    out.band_cap = band_cap;
    // (80 registers only where shared memory leaves room for more than the
    // 16 warps per SM of the 128-register kernel.)
    const bool more_warps =
        17 * (region_bytes_for_stage(stage, stage == kStageGlobal ? 0 : max_n_here) + tb) +
            2 * 1024 <= (int)P->prop.sharedMemPerMultiprocessor;
    const int reg_class = choice && choice->set ? choice->reg_class
                          : (untuned_global && stage != kStageBand && more_warps) ? 1
                                                                                   : 0;
    const int variant = kernel_variant(kind, stage, reg_class);
    out.stage = stage;
    if (choice && choice->set) {
        // The autotuner's measured configuration (a persistent launch takes
        // items from its queue; a plain one strides over them statically).
        const int w = choice->warps_per_cta;
        if (w < 1 || w > kMaxThreadsPerCta / 32 || (int64_t)w * region > smem_blk)
            return set_err(err, errlen, B200SA_EINVAL, "tuned shape does not fit");
        int ctas = 0;
        int rc = occupancy(P, variant, w, region, &ctas, err, errlen);
        if (rc) return rc;
        if (ctas < 1) return set_err(err, errlen, B200SA_ECUDA, "tuned shape does not fit on an SM");
        if (choice->ctas_per_sm > 0) ctas = std::min(ctas, choice->ctas_per_sm);
        int wl = w;
        if (!persistent) {
            // One problem's reads: spread them over every SM first, as the
            // occupancy rule does (a tuned CTA width assumes a full bucket).
            const int sms = P->prop.multiProcessorCount;
            wl = (int)std::min<int64_t>(w, std::max<int64_t>(1, (items + sms - 1) / sms));
            if (wl != w) {
                int rc = occupancy(P, variant, wl, region, &ctas, err, errlen);
                if (rc) return rc;
                if (choice->ctas_per_sm > 0) ctas = std::min(ctas, choice->ctas_per_sm * w / wl);
            }
        }
        out.cap_n = cap;
        out.warps_per_cta = wl;
        out.region = region;
        out.grid = (int)std::max<int64_t>(
            1, std::min<int64_t>((int64_t)P->prop.multiProcessorCount * ctas, (items + wl - 1) / wl));
        out.variant = variant;
        return B200SA_OK;
    }
    int best_w = 1, best_warps = 0;
    for (int w = 1; w <= kMaxThreadsPerCta / 32; ++w) {
        if ((int64_t)w * region > smem_blk) break;
        int ctas = 0;
        int rc = occupancy(P, variant, w, region, &ctas, err, errlen);
        if (rc) return rc;
        if (ctas * w > best_warps) {
            best_warps = ctas * w;
            best_w = w;
        }
    }
    if (best_warps == 0)
        return set_err(err, errlen, B200SA_ECUDA, "kernel does not fit on an SM");
    // Fewer items than resident warp slots: spread them over every SM first.
    const int sms = P->prop.multiProcessorCount;
    int w = (int)std::min<int64_t>(best_w, std::max<int64_t>(1, (items + sms - 1) / sms));
    int grid;
    if (persistent) {
        int ctas = best_warps / best_w;
        if (w != best_w) {
            int rc = occupancy(P, variant, w, region, &ctas, err, errlen);
            if (rc) return rc;
        }
        grid = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)sms * ctas, (items + w - 1) / w));
    } else {
        grid = (int)std::max<int64_t>(1, (items + w - 1) / w);
    }
    out.cap_n = cap;
    out.warps_per_cta = w;
    out.region = region;
    out.grid = grid;
    out.variant = variant;
    return B200SA_OK;
}

int ensure_scratch(b200sa_plan_s *P, int64_t slots, int64_t stride, char *err,
                   size_t errlen) {
    stride = (stride + 15) & ~int64_t(15);
    if (slots <= P->scratch_slots && stride <= P->scratch_stride) return B200SA_OK;
    slots = std::max(slots, P->scratch_slots);
    stride = std::max(stride, P->scratch_stride);
    // The old slots may still be in use by an enqueued run, and a captured
    // graph holds their addresses.
    B200SA_CUDA(cudaDeviceSynchronize());
    if (P->graph_exec) {
        cudaGraphExecDestroy(P->graph_exec);
        P->graph_exec = nullptr;
    }
    B200SA_CUDA(P->scratch_de.alloc((size_t)(slots * stride)));
    B200SA_CUDA(P->scratch_s.alloc((size_t)(slots * stride)));
    P->scratch_slots = slots;
    P->scratch_stride = stride;
    return B200SA_OK;
}

LaunchArgs base_args(b200sa_plan_s *P, const int8_t *in, int8_t *out, double *en,
                     const uint64_t *seeds) {
    LaunchArgs a{};
    a.problems = P->dprobs.ptr;
    a.states_in = in;
    a.states_out = out;
    a.energies = en;
    a.seeds = seeds ? seeds : P->dseeds.ptr;
    a.stats = P->dstats.ptr;
    return a;
}

// One launch over `count` items.  Persistent launches take items from the
// work-queue head `qhead` (zeroed by the caller, stream-ordered).
int items_shape(b200sa_plan_s *P, int kind, int32_t max_n_here, int64_t count, bool persistent,
                bool shared_stream, const TuneChoice *choice, LaunchShape &s, char *err,
                size_t errlen, int band_w_here = 0) {
    int rc = shape_for(P, kind, max_n_here, shared_stream ? 1 : count,
                       persistent && !shared_stream, s, err, errlen,
                       shared_stream ? nullptr : choice, band_w_here);
    if (rc) return rc;
    if (shared_stream) {  // one stream continued read after read: one warp
        s.grid = 1;
        s.warps_per_cta = 1;
    }
    return B200SA_OK;
}

int launch_shape(b200sa_plan_s *P, LaunchArgs a, const LaunchShape &s, const int64_t *items,
                 int64_t count, int32_t max_n_here, bool persistent, bool shared_stream,
                 unsigned long long *qhead, int64_t slot0, cudaStream_t st, char *err,
                 size_t errlen) {
    if (count <= 0) return B200SA_OK;
    if (s.stage != kStageShared) {
        const int64_t end = slot0 + (int64_t)s.grid * s.warps_per_cta;
        if (end > P->scratch_slots || max_n_here > P->scratch_stride)
            return set_err(err, errlen, B200SA_EINVAL, "internal: global slots not reserved");
        a.scratch_de = P->scratch_de.ptr + slot0 * P->scratch_stride;
        a.scratch_s = P->scratch_s.ptr + slot0 * P->scratch_stride;
        a.scratch_stride = P->scratch_stride;
        a.num_slots = end - slot0;
    }
    a.items = items;
    a.num_items = count;
    a.smem_cap_n = s.cap_n;
    a.touch_bytes = s.touch_bytes;
    a.band_cap = s.band_cap;
    a.queue_head = (persistent && !shared_stream) ? qhead : nullptr;
    B200SA_CUDA(launch_sa(s.variant, a, s.grid, s.warps_per_cta, s.region, st));
    P->launches++;
    return B200SA_OK;
}

int launch_items(b200sa_plan_s *P, LaunchArgs a, int kind, const int64_t *items,
                 int64_t count, int32_t max_n_here, bool persistent, bool shared_stream,
                 unsigned long long *qhead, cudaStream_t st, char *err, size_t errlen,
                 const TuneChoice *choice, int band_w_here) {
    if (count <= 0) return B200SA_OK;
    LaunchShape s{};
    int rc = items_shape(P, kind, max_n_here, count, persistent, shared_stream, choice, s, err,
                         errlen, band_w_here);
    if (rc) return rc;
    if (s.stage != kStageShared) {
        rc = ensure_scratch(P, (int64_t)s.grid * s.warps_per_cta, max_n_here, err, errlen);
        if (rc) return rc;
    }
    return launch_shape(P, a, s, items, count, max_n_here, persistent, shared_stream, qhead, 0,
                        st, err, errlen);
}

int collect_stats(b200sa_plan_s *P, const std::vector<std::pair<int, int>> &ranges,
                  b200sa_stats *stats, char *err, size_t errlen) {
    // ranges: (problem, reads completed from read 0)
    if (!stats) return B200SA_OK;
    std::vector<ReadStats> hs((size_t)P->total_reads);
    if (P->total_reads)
        B200SA_CUDA(cudaMemcpy(hs.data(), P->dstats.ptr,
                               sizeof(ReadStats) * (size_t)P->total_reads,
                               cudaMemcpyDeviceToHost));
    for (auto &pr : ranges) {
        const int p = pr.first;
        const int64_t att_per_read = (int64_t)P->n[p] * P->sweeps[p];
        for (int r = 0; r < pr.second; ++r) {
            const size_t rd = (size_t)(P->read_off[p] + r);
            const ReadStats &x = hs[rd];
            if (stats->read_near_ties) stats->read_near_ties[rd] = x.near_ties;
            stats->flips += (int64_t)x.flips;
            stats->passes += (int64_t)x.passes;
            stats->near_ties += (int64_t)x.near_ties;
            stats->attempts += att_per_read;
            stats->reads += 1;
        }
    }
    return B200SA_OK;
}

// Persistent mode: one launch per non-empty bucket, spread over forked
// streams, the bucket with the longest items first so later buckets fill SMs
// as earlier ones drain.
int run_persistent(b200sa_plan_s *P, LaunchArgs a, cudaStream_t st, char *err,
                   size_t errlen) {
    // Shapes first: the launches below may run at the same time, so those
    // that keep their state in global slots get disjoint slot ranges.
    LaunchShape shape[kBuckets];
    int64_t slot0[kBuckets] = {};
    int64_t slots = 0;
    int32_t stride = 0;
    for (int b = 0; b < kBuckets; ++b) {
        const int64_t cnt = P->bucket_off[b + 1] - P->bucket_off[b];
        if (cnt <= 0) continue;
        int rc = items_shape(P, b % kKinds, P->bucket_max_n[b], cnt, true, false, &P->tune[b],
                             shape[b], err, errlen, P->bucket_band_w[b]);
        if (rc) return rc;
        if (shape[b].stage != kStageShared) {
            slot0[b] = slots;
            slots += (int64_t)shape[b].grid * shape[b].warps_per_cta;
            stride = std::max(stride, P->bucket_max_n[b]);
        }
    }
    if (slots > 0) {
        int rc = ensure_scratch(P, slots, stride, err, errlen);
        if (rc) return rc;
    }
    if (P->dry_run) return B200SA_OK;
    B200SA_CUDA(cudaMemsetAsync(P->qhead.ptr, 0, sizeof(unsigned long long) * kBuckets, st));
    B200SA_CUDA(cudaEventRecord(P->fork, st));
    int order[kBuckets];
    for (int b = 0; b < kBuckets; ++b) order[b] = b;
    std::stable_sort(order, order + kBuckets, [&](int x, int y) {
        return P->bucket_lead_cost[x] > P->bucket_lead_cost[y];
    });
    bool used[kStreams] = {};
    int next = 0;
    for (int i = 0; i < kBuckets; ++i) {
        const int b = order[i];
        const int64_t cnt = P->bucket_off[b + 1] - P->bucket_off[b];
        P->bucket_timed[b] = cnt > 0;
        if (cnt <= 0) continue;
        const int si = next++ % kStreams;
        if (!used[si]) B200SA_CUDA(cudaStreamWaitEvent(P->bstream[si], P->fork, 0));
        used[si] = true;
        // Inside a capture the timing events become event-record nodes of the
        // graph (external records), so every replay records them.
        const unsigned evflags = P->capturing ? cudaEventRecordExternal : cudaEventRecordDefault;
        B200SA_CUDA(cudaEventRecordWithFlags(P->bev[b][0], P->bstream[si], evflags));
        int rc = launch_shape(P, a, shape[b], P->items_lpt.ptr + P->bucket_off[b], cnt,
                              P->bucket_max_n[b], true, false, P->qhead.ptr + b, slot0[b],
                              P->bstream[si], err, errlen);
        if (rc) return rc;
        B200SA_CUDA(cudaEventRecordWithFlags(P->bev[b][1], P->bstream[si], evflags));
        P->bshape[b] = shape[b];
    }
    for (int si = 0; si < kStreams; ++si) {
        if (!used[si]) continue;
        B200SA_CUDA(cudaEventRecord(P->join[si], P->bstream[si]));
        B200SA_CUDA(cudaStreamWaitEvent(st, P->join[si], 0));
    }
    return B200SA_OK;
}

}  // namespace host
}  // namespace b200sa

extern "C" {

const char *b200sa_version(void) { return "b200sa 0.6.0 (sm_100a)"; }

int b200sa_check_acceptance(int64_t samples, uint64_t seed, int32_t device,
                            int64_t counts[6], char *err, size_t errlen) {
    if (!counts || samples < 0) return set_err(err, errlen, B200SA_EINVAL, "bad arguments");
    DeviceGuard guard;
    cudaDeviceProp prop;
    int rc = select_device(device, prop, err, errlen);
    if (rc) return rc;
    DevArray<unsigned long long> d;
    B200SA_CUDA(d.alloc(6));
    B200SA_CUDA(cudaMemset(d.ptr, 0, 6 * sizeof(unsigned long long)));
    B200SA_CUDA(acceptance_check(samples, seed, d.ptr));
    unsigned long long h[6];
    B200SA_CUDA(cudaMemcpy(h, d.ptr, sizeof(h), cudaMemcpyDeviceToHost));
    for (int i = 0; i < 6; ++i) counts[i] = (int64_t)h[i];
    return B200SA_OK;
}

int b200sa_plan_create(const b200sa_problem *problems, int32_t num_problems,
                       int32_t device, b200sa_plan *out, char *err, size_t errlen) {
    if (!out) return set_err(err, errlen, B200SA_EINVAL, "out is NULL");
    *out = nullptr;
    if (num_problems < 0 || (num_problems > 0 && !problems))
        return set_err(err, errlen, B200SA_EINVAL, "bad problem list");
    for (int32_t i = 0; i < num_problems; ++i) {
        std::string msg;
        const int rc = validate_problem(problems[i], msg);
        if (rc) return set_err(err, errlen, rc, "problem " + std::to_string(i) + ": " + msg);
        if (problems[i].num_reads > 0 && problems[i].num_vars > 0 && !problems[i].seeds)
            return set_err(err, errlen, B200SA_EINVAL,
                           "problem " + std::to_string(i) + ": seeds is NULL");
    }
    DeviceGuard guard;
    std::unique_ptr<b200sa_plan_s> P(new b200sa_plan_s());
    int rc = select_device(device, P->prop, err, errlen);
    if (rc) return rc;
    P->device = device;
    B200SA_CUDA(cudaStreamCreateWithFlags(&P->stream, cudaStreamNonBlocking));
    for (int b = 0; b < kStreams; ++b) {
        B200SA_CUDA(cudaStreamCreateWithFlags(&P->bstream[b], cudaStreamNonBlocking));
        B200SA_CUDA(cudaEventCreateWithFlags(&P->join[b], cudaEventDisableTiming));
    }
    B200SA_CUDA(cudaEventCreate(&P->ev0));
    B200SA_CUDA(cudaEventCreate(&P->ev1));
    B200SA_CUDA(cudaEventCreateWithFlags(&P->fork, cudaEventDisableTiming));
    for (int b = 0; b < kBuckets; ++b)
        for (int k = 0; k < 2; ++k) B200SA_CUDA(cudaEventCreate(&P->bev[b][k]));
    P->num_problems = num_problems;
    // On chip when at least three warps' regions fit in one SM.
    {
        const int smem_sm = (int)P->prop.sharedMemPerMultiprocessor;
        int lo = 0, hi = 1 << 20;
        while (lo < hi) {
            const int mid = (lo + hi + 1) / 2;
            if (3 * region_bytes_for(mid) + 3 * 1024 <= smem_sm) lo = mid; else hi = mid - 1;
        }
        P->onchip_max = lo;
        lo = 0, hi = 1 << 20;
        while (lo < hi) {
            const int mid = (lo + hi + 1) / 2;
            if (24 * region_bytes_for(mid) + 2 * 1024 <= smem_sm) lo = mid; else hi = mid - 1;
        }
        P->onchip_fast = lo;
    }

    // Pack and lay out every problem in one device arena.
    std::vector<PackedAdjacency> adj((size_t)num_problems);
    std::vector<ArenaOffsets> off((size_t)num_problems);
    size_t bytes = 0;
    auto take = [&](size_t sz) {
        const size_t o = bytes;
        bytes = align16(bytes + sz);
        return o;
    };
    P->state_off.assign((size_t)num_problems + 1, 0);
    P->read_off.assign((size_t)num_problems + 1, 0);
    // The problems' adjacency is packed on up to 32 host threads (problems
    // are independent; each thread takes the next unpacked one).
    {
        const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
        const int nt = std::min(std::min(hw, 32), (int)num_problems);
        std::atomic<int32_t> next{0};
        std::atomic<bool> failed{false};
        auto work = [&]() {
            for (int32_t i; (i = next.fetch_add(1)) < num_problems;) {
                try {
                    pack_adjacency(problems[i], adj[i]);
                } catch (...) {
                    failed = true;
                }
            }
        };
        if (nt <= 1) {
            work();
        } else {
            std::vector<std::thread> pool;
            for (int t = 0; t < nt; ++t) pool.emplace_back(work);
            for (std::thread &t : pool) t.join();
        }
        if (failed) return set_err(err, errlen, B200SA_ENOMEM, "out of host memory packing problems");
    }
    for (int32_t i = 0; i < num_problems; ++i) {
        const b200sa_problem &q = problems[i];
        const size_t n = (size_t)q.num_vars, m = (size_t)q.num_couplers,
                     nb = (size_t)q.num_betas;
        ArenaOffsets &o = off[i];
        o.vinfo = take(8 * n);
        o.dist = take(n);
        o.share = take(4 * n);
        o.col = take(4 * 2 * m);
        o.w = take(8 * 2 * m);
        o.h = take(8 * n);
        o.cu = take(4 * m);
        o.cv = take(4 * m);
        o.cw = take(8 * m);
        o.betas = take(8 * nb);
        o.thr = take(8 * nb);
        o.back = take(8 * n);
        o.bw = take(8 * adj[i].bw.size());
        o.dw = take(8 * adj[i].dense_w.size());
        o.dbits = take(4 * adj[i].dense_bits.size());
        P->state_off[i + 1] = P->state_off[i] + (int64_t)q.num_reads * q.num_vars;
        P->read_off[i + 1] = P->read_off[i] + q.num_reads;
        P->n.push_back(q.num_vars);
        P->reads.push_back(q.num_reads);
        P->sweeps.push_back(q.sweeps_per_beta * q.num_betas);
        P->max_n = std::max(P->max_n, q.num_vars);
    }
    P->total_state = P->state_off[num_problems];
    P->total_reads = P->read_off[num_problems];
    std::vector<uint8_t> staging(bytes);
    for (int32_t i = 0; i < num_problems; ++i) {
        const b200sa_problem &q = problems[i];
        const ArenaOffsets &o = off[i];
        const size_t n = (size_t)q.num_vars, m = (size_t)q.num_couplers,
                     nb = (size_t)q.num_betas;
        if (m) {
            std::memcpy(&staging[o.col], adj[i].col.data(), 4 * 2 * m);
            std::memcpy(&staging[o.w], adj[i].w.data(), 8 * 2 * m);
            std::memcpy(&staging[o.cu], q.coupler_starts, 4 * m);
            std::memcpy(&staging[o.cv], q.coupler_ends, 4 * m);
            std::memcpy(&staging[o.cw], q.coupler_weights, 8 * m);
        }
        if (n) {
            std::memcpy(&staging[o.vinfo], adj[i].vinfo.data(), 8 * n);
            std::memcpy(&staging[o.dist], adj[i].dist.data(), n);
            std::memcpy(&staging[o.share], adj[i].share.data(), 4 * n);
            std::memcpy(&staging[o.h], q.h, 8 * n);
            std::memcpy(&staging[o.back], adj[i].back.data(), 8 * n);
        }
        if (!adj[i].bw.empty())
            std::memcpy(&staging[o.bw], adj[i].bw.data(), 8 * adj[i].bw.size());
        if (!adj[i].dense_w.empty()) {
            std::memcpy(&staging[o.dw], adj[i].dense_w.data(), 8 * adj[i].dense_w.size());
            std::memcpy(&staging[o.dbits], adj[i].dense_bits.data(), 4 * adj[i].dense_bits.size());
        }
        if (nb) {
            std::memcpy(&staging[o.betas], q.beta_schedule, 8 * nb);
            double *thr = reinterpret_cast<double *>(&staging[o.thr]);
            // cpu_sa.cpp:131, evaluated once per beta on the host (IEEE division).
            for (size_t b = 0; b < nb; ++b) thr[b] = 44.36142 / q.beta_schedule[b];
        }
    }
    B200SA_CUDA(P->arena.alloc(std::max<size_t>(bytes, 16)));
    if (bytes)
        B200SA_CUDA(cudaMemcpyAsync(P->arena.ptr, staging.data(), bytes,
                                    cudaMemcpyHostToDevice, P->stream));
    P->offs = off;
    P->rows.resize((size_t)num_problems);
    P->bw_src.resize((size_t)num_problems);
    for (int32_t i = 0; i < num_problems; ++i) P->rows[i] = std::move(adj[i].row);
    P->hprobs.resize((size_t)num_problems);
    for (int32_t i = 0; i < num_problems; ++i) {
        const b200sa_problem &q = problems[i];
        const ArenaOffsets &o = off[i];
        ProblemDev &d = P->hprobs[i];
        uint8_t *base = P->arena.ptr;
        d.n = q.num_vars;
        d.sweeps_per_beta = q.sweeps_per_beta;
        d.num_betas = q.num_betas;
        d.num_reads = q.num_reads;
        d.m = q.num_couplers;
        d.state_offset = P->state_off[i];
        d.read_offset = P->read_off[i];
        d.vinfo = reinterpret_cast<const uint2 *>(base + o.vinfo);
        d.dist = base + o.dist;
        d.share = reinterpret_cast<const uint32_t *>(base + o.share);
        d.col = reinterpret_cast<const int32_t *>(base + o.col);
        d.w = reinterpret_cast<const double *>(base + o.w);
        d.h = reinterpret_cast<const double *>(base + o.h);
        d.cu = reinterpret_cast<const int32_t *>(base + o.cu);
        d.cv = reinterpret_cast<const int32_t *>(base + o.cv);
        d.cw = reinterpret_cast<const double *>(base + o.cw);
        d.betas = reinterpret_cast<const double *>(base + o.betas);
        d.thresholds = reinterpret_cast<const double *>(base + o.thr);
        d.varorder = q.varorder;
        d.proposal = q.proposal;
        d.regular_degree = adj[i].regular_degree;
        d.regular_magic = d.regular_degree ? (65536u + (uint32_t)d.regular_degree - 1) /
                                                 (uint32_t)d.regular_degree
                                           : 0u;
        d.resolve = (adj[i].resolve && resolve_allowed()) ? 1 : 0;
        d.dense = (d.resolve && adj[i].dense && dense_allowed()) ? 1 : 0;
        d.back = reinterpret_cast<const uint2 *>(base + o.back);
        d.bw = reinterpret_cast<const double *>(base + o.bw);
        d.dense_w = reinterpret_cast<const double *>(base + o.dw);
        d.dense_bits = reinterpret_cast<const uint32_t *>(base + o.dbits);
        d.band_b = adj[i].band_b;
        d.band_w = band_allowed() ? adj[i].band_w : 0;
        P->bw_src[i] = std::move(adj[i].bw_src);
    }
    B200SA_CUDA(P->dprobs.alloc((size_t)std::max(num_problems, 1)));
    if (num_problems)
        B200SA_CUDA(cudaMemcpyAsync(P->dprobs.ptr, P->hprobs.data(),
                                    sizeof(ProblemDev) * (size_t)num_problems,
                                    cudaMemcpyHostToDevice, P->stream));

    // Seeds and work items: plain order (problem, read) and, for the
    // persistent mode, grouped by size bucket, longest first inside a bucket.
    std::vector<uint64_t> seeds((size_t)P->total_reads);
    std::vector<int64_t> plain;
    plain.reserve((size_t)P->total_reads);
    P->plain_item_off.assign((size_t)num_problems + 1, 0);
    for (int32_t i = 0; i < num_problems; ++i) {
        const b200sa_problem &q = problems[i];
        P->plain_item_off[i] = (int64_t)plain.size();
        if (q.num_vars == 0) continue;  // nothing to anneal; energies are zero
        for (int32_t r = 0; r < q.num_reads; ++r) {
            seeds[(size_t)(P->read_off[i] + r)] = q.seeds[r];
            plain.push_back(((int64_t)i << 32) | (int64_t)r);
        }
    }
    P->plain_item_off[num_problems] = (int64_t)plain.size();
    auto cost = [&](int64_t it) {
        const int p = (int)(it >> 32);
        return (int64_t)P->n[p] * P->sweeps[p];
    };
    auto bucket_of = [&](int64_t it) {
        const int p = (int)(it >> 32);
        return size_class(P->n[p], P->onchip_max) * kKinds + kind_of(P->hprobs[p]);
    };
    std::vector<int64_t> lpt = plain;
    std::stable_sort(lpt.begin(), lpt.end(), [&](int64_t x, int64_t y) {
        const int bx = bucket_of(x), by = bucket_of(y);
        if (bx != by) return bx < by;
        return cost(x) > cost(y);
    });
    for (int b = 0; b <= kBuckets; ++b) P->bucket_off[b] = 0;
    for (int64_t it : lpt) {
        const int p = (int)(it >> 32);
        const int b = bucket_of(it);
        P->bucket_off[b + 1]++;
        P->bucket_max_n[b] = std::max(P->bucket_max_n[b], P->n[p]);
        P->bucket_lead_cost[b] = std::max(P->bucket_lead_cost[b], cost(it));
    }
    for (int b = 0; b < kBuckets; ++b) P->bucket_off[b + 1] += P->bucket_off[b];
    // A bucket may use the band location when all of its problems are banded.
    {
        bool all[kBuckets];
        for (int b = 0; b < kBuckets; ++b) all[b] = true;
        for (int64_t it : lpt) {
            const int p = (int)(it >> 32);
            const int b = bucket_of(it);
            const int32_t w = P->hprobs[p].band_w;
            if (w == 0) all[b] = false;
            P->bucket_band_w[b] = std::max(P->bucket_band_w[b], w);
        }
        for (int b = 0; b < kBuckets; ++b)
            if (!all[b]) P->bucket_band_w[b] = 0;
    }

    B200SA_CUDA(P->dseeds.alloc(std::max<size_t>(seeds.size(), 1)));
    B200SA_CUDA(P->dstats.alloc(std::max<size_t>(seeds.size(), 1)));
    B200SA_CUDA(P->items_plain.alloc(std::max<size_t>(plain.size(), 1)));
    B200SA_CUDA(P->items_lpt.alloc(std::max<size_t>(lpt.size(), 1)));
    B200SA_CUDA(P->qhead.alloc(kBuckets));
    if (!seeds.empty())
        B200SA_CUDA(cudaMemcpyAsync(P->dseeds.ptr, seeds.data(), 8 * seeds.size(),
                                    cudaMemcpyHostToDevice, P->stream));
    if (!plain.empty()) {
        B200SA_CUDA(cudaMemcpyAsync(P->items_plain.ptr, plain.data(), 8 * plain.size(),
                                    cudaMemcpyHostToDevice, P->stream));
        B200SA_CUDA(cudaMemcpyAsync(P->items_lpt.ptr, lpt.data(), 8 * lpt.size(),
                                    cudaMemcpyHostToDevice, P->stream));
    }
    B200SA_CUDA(upload_jump_table(jump_table(), P->stream));
    B200SA_CUDA(cudaStreamSynchronize(P->stream));
    P->h_items_lpt = std::move(lpt);
    *out = P.release();
    return B200SA_OK;
}

int b200sa_plan_layout(b200sa_plan plan, int64_t *state_offsets, int64_t *read_offsets) {
    if (!plan) return B200SA_EINVAL;
    for (int i = 0; i <= plan->num_problems; ++i) {
        if (state_offsets) state_offsets[i] = plan->state_off[i];
        if (read_offsets) read_offsets[i] = plan->read_off[i];
    }
    return B200SA_OK;
}

int b200sa_plan_destroy(b200sa_plan plan) {
    if (!plan) return B200SA_OK;
    DeviceGuard guard;
    cudaSetDevice(plan->device);
    cudaDeviceSynchronize();
    delete plan;
    return B200SA_OK;
}

int b200sa_plan_run(b200sa_plan plan, int32_t mode, const int8_t *d_states_in,
                    int8_t *d_states_out, double *d_energies, const uint64_t *d_seeds,
                    void *stream, int32_t sync, b200sa_stats *stats, char *err,
                    size_t errlen) {
    if (!plan) return set_err(err, errlen, B200SA_EINVAL, "plan is NULL");
    if (mode != B200SA_MODE_PERSISTENT && mode != B200SA_MODE_PLAIN && mode != B200SA_MODE_GRAPH &&
        mode != B200SA_MODE_PLAIN_TUNED)
        return set_err(err, errlen, B200SA_EINVAL, "unknown mode");
    if (plan->total_reads > 0 && (!d_states_in || !d_states_out || !d_energies))
        return set_err(err, errlen, B200SA_EINVAL, "device buffers are NULL");
    DeviceGuard guard;
    B200SA_CUDA(cudaSetDevice(plan->device));
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : plan->stream;
    reset_stats(stats);
    LaunchArgs a = base_args(plan, d_states_in, d_states_out, d_energies, d_seeds);
    plan->launches = 0;
    // Problems with no variables: energies are 0 (cpu_sa.cpp:217-226 over nothing).
    for (int i = 0; i < plan->num_problems; ++i) {
        if (plan->n[i] == 0 && plan->reads[i] > 0)
            B200SA_CUDA(cudaMemsetAsync(d_energies + plan->read_off[i], 0,
                                        sizeof(double) * (size_t)plan->reads[i], st));
    }
    B200SA_CUDA(cudaEventRecord(plan->ev0, st));
    int rc = B200SA_OK;
    if (mode == B200SA_MODE_PERSISTENT) {
        rc = run_persistent(plan, a, st, err, errlen);
    } else if (mode == B200SA_MODE_GRAPH) {
        rc = run_graph(plan, a, st, err, errlen);
    } else {
        // One launch per problem; PLAIN_TUNED gives each launch the tuned
        // shape of the problem's bucket (its size class and kind).
        const bool tuned = mode == B200SA_MODE_PLAIN_TUNED;
        for (int i = 0; i < plan->num_problems && rc == B200SA_OK; ++i) {
            const int64_t o = plan->plain_item_off[i];
            const int kind = kind_of(plan->hprobs[i]);
            const TuneChoice *choice =
                tuned ? &plan->tune[size_class(plan->n[i], plan->onchip_max) * kKinds + kind]
                      : nullptr;
            rc = launch_items(plan, a, kind, plan->items_plain.ptr + o,
                              plan->plain_item_off[i + 1] - o, plan->n[i], false, false,
                              nullptr, st, err, errlen, choice, plan->hprobs[i].band_w);
        }
    }
    if (rc) return rc;
    B200SA_CUDA(cudaEventRecord(plan->ev1, st));
    if (sync) {
        B200SA_CUDA(cudaStreamSynchronize(st));
        if (stats) {
            float ms = 0.f;
            B200SA_CUDA(cudaEventElapsedTime(&ms, plan->ev0, plan->ev1));
            std::vector<std::pair<int, int>> ranges;
            for (int i = 0; i < plan->num_problems; ++i)
                ranges.emplace_back(i, plan->n[i] ? plan->reads[i] : 0);
            rc = collect_stats(plan, ranges, stats, err, errlen);
            if (rc) return rc;
            for (int i = 0; i < plan->num_problems; ++i) {
                if (plan->n[i] != 0) continue;
                stats->reads += plan->reads[i];
                if (stats->read_near_ties)
                    for (int r = 0; r < plan->reads[i]; ++r)
                        stats->read_near_ties[plan->read_off[i] + r] = 0;
            }
            stats->kernel_ms = ms;
            stats->launches = plan->launches;
        }
    }
    return B200SA_OK;
}

int b200sa_sample_batch(const b200sa_problem *problems, int32_t num_problems, int32_t mode,
                        int32_t device, b200sa_stats *stats, char *err, size_t errlen) {
    for (int i = 0; i < num_problems && problems; ++i) {
        const size_t sz = (size_t)problems[i].num_reads * (size_t)problems[i].num_vars;
        if (sz && !problems[i].states)
            return set_err(err, errlen, B200SA_EINVAL,
                           "problem " + std::to_string(i) + ": states is NULL");
        if (problems[i].num_reads > 0 && !problems[i].energies)
            return set_err(err, errlen, B200SA_EINVAL,
                           "problem " + std::to_string(i) + ": energies is NULL");
    }
    b200sa_plan plan = nullptr;
    int rc = b200sa_plan_create(problems, num_problems, device, &plan, err, errlen);
    if (rc) return rc;
    std::unique_ptr<b200sa_plan_s, int (*)(b200sa_plan)> hold(plan, b200sa_plan_destroy);
    const char *cache = std::getenv("B200SA_TUNE_CACHE");
    if (cache && *cache && mode != B200SA_MODE_PLAIN) {
        rc = b200sa_plan_autotune(plan, cache, 0, nullptr, 0, err, errlen);
        if (rc < 0) return rc;
    }
    DeviceGuard guard;
    B200SA_CUDA(cudaSetDevice(plan->device));
    DevArray<int8_t> dstates;
    DevArray<double> den;
    B200SA_CUDA(dstates.alloc((size_t)std::max<int64_t>(plan->total_state, 1)));
    B200SA_CUDA(den.alloc((size_t)std::max<int64_t>(plan->total_reads, 1)));
    for (int i = 0; i < num_problems; ++i) {
        const size_t sz = (size_t)problems[i].num_reads * (size_t)problems[i].num_vars;
        if (sz)
            B200SA_CUDA(cudaMemcpyAsync(dstates.ptr + plan->state_off[i], problems[i].states,
                                        sz, cudaMemcpyHostToDevice, plan->stream));
    }
    rc = b200sa_plan_run(plan, mode, dstates.ptr, dstates.ptr, den.ptr, nullptr, nullptr, 1,
                         stats, err, errlen);
    if (rc) return rc;
    for (int i = 0; i < num_problems; ++i) {
        const size_t sz = (size_t)problems[i].num_reads * (size_t)problems[i].num_vars;
        if (sz)
            B200SA_CUDA(cudaMemcpyAsync(problems[i].states, dstates.ptr + plan->state_off[i],
                                        sz, cudaMemcpyDeviceToHost, plan->stream));
        if (problems[i].num_reads)
            B200SA_CUDA(cudaMemcpyAsync(problems[i].energies, den.ptr + plan->read_off[i],
                                        sizeof(double) * (size_t)problems[i].num_reads,
                                        cudaMemcpyDeviceToHost, plan->stream));
    }
    B200SA_CUDA(cudaStreamSynchronize(plan->stream));
    return (int)std::min<int64_t>(plan->total_reads, INT32_MAX);
}

int b200sa_sample(int32_t num_vars, const double *h, int64_t num_couplers,
                  const int32_t *coupler_starts, const int32_t *coupler_ends,
                  const double *coupler_weights, int32_t num_reads, int8_t *states,
                  double *energies, int32_t sweeps_per_beta, int32_t num_betas,
                  const double *beta_schedule, const uint64_t *seeds, int32_t num_seeds,
                  int32_t varorder, int32_t proposal, b200sa_interrupt_fn interrupt_fn,
                  void *interrupt_ctx, int32_t device, b200sa_stats *stats, char *err,
                  size_t errlen) {
    reset_stats(stats);
    if (num_reads < 0) return set_err(err, errlen, B200SA_EINVAL, "num_reads < 0");
    if (num_reads == 0) return 0;
    if (!states && num_vars > 0)
        return set_err(err, errlen, B200SA_EINVAL, "states is NULL");
    if (!energies) return set_err(err, errlen, B200SA_EINVAL, "energies is NULL");
    if (!seeds || (num_seeds != 1 && num_seeds != num_reads))
        return set_err(err, errlen, B200SA_EINVAL,
                       "num_seeds must be 1 (one continued stream) or num_reads (per read)");
    const bool shared = num_seeds == 1 && num_reads > 1;
    b200sa_problem q{};
    q.num_vars = num_vars;
    q.h = h;
    q.num_couplers = num_couplers;
    q.coupler_starts = coupler_starts;
    q.coupler_ends = coupler_ends;
    q.coupler_weights = coupler_weights;
    q.num_reads = num_reads;
    q.states = states;
    q.energies = energies;
    q.sweeps_per_beta = sweeps_per_beta;
    q.num_betas = num_betas;
    q.beta_schedule = beta_schedule;
    std::vector<uint64_t> shared_seeds;
    if (shared) {  // the kernel seeds only the first read and continues the stream
        shared_seeds.assign((size_t)num_reads, seeds[0]);
        q.seeds = shared_seeds.data();
    } else {
        q.seeds = seeds;
    }
    q.varorder = varorder;
    q.proposal = proposal;
    if (num_vars == 0) {  // cpu_sa.cpp: every read's energy sums nothing
        std::string msg;
        int rc = validate_problem(q, msg);
        if (rc) return set_err(err, errlen, rc, msg);
        for (int32_t r = 0; r < num_reads; ++r) {
            energies[r] = 0.0;
            if (stats && stats->read_near_ties) stats->read_near_ties[r] = 0;
            if (interrupt_fn && interrupt_fn(interrupt_ctx)) {
                if (stats) stats->reads = r + 1;
                return r + 1;
            }
        }
        if (stats) stats->reads = num_reads;
        return num_reads;
    }
    b200sa_plan plan = nullptr;
    int rc = b200sa_plan_create(&q, 1, device, &plan, err, errlen);
    if (rc) return rc;
    std::unique_ptr<b200sa_plan_s, int (*)(b200sa_plan)> hold(plan, b200sa_plan_destroy);
    DeviceGuard guard;
    B200SA_CUDA(cudaSetDevice(plan->device));
    const size_t n = (size_t)num_vars;
    DevArray<int8_t> dstates;
    DevArray<double> den;
    B200SA_CUDA(dstates.alloc(n * (size_t)num_reads));
    B200SA_CUDA(den.alloc((size_t)num_reads));
    B200SA_CUDA(cudaMemcpyAsync(dstates.ptr, states, n * (size_t)num_reads,
                                cudaMemcpyHostToDevice, plan->stream));
    if (shared) B200SA_CUDA(plan->carry.alloc(kCarryWords));

    // Chunks: everything at once without an interrupt; with one, a resident
    // wave of reads (per-read seeds) or one read (continued stream) per launch,
    // polling the callback after each completed read in read order.
    int64_t chunk = num_reads;
    if (interrupt_fn) {
        if (shared) {
            chunk = 1;
        } else {
            LaunchShape s{};
            rc = shape_for(plan, kind_of(plan->hprobs[0]), num_vars, num_reads, true, s, err,
                           errlen, nullptr, plan->hprobs[0].band_w);
            if (rc) return rc;
            int ctas = 0;
            rc = occupancy(plan, s.variant, s.warps_per_cta, s.region, &ctas, err, errlen);
            if (rc) return rc;
            chunk = std::max<int64_t>(
                1, (int64_t)plan->prop.multiProcessorCount * ctas * s.warps_per_cta);
        }
    }
    LaunchArgs a = base_args(plan, dstates.ptr, dstates.ptr, den.ptr, nullptr);
    a.rng_carry = plan->carry.ptr;
    a.shared_stream = shared ? 1 : 0;
    float total_ms = 0.f;
    int32_t done = 0;
    bool stop = false;
    while (done < num_reads && !stop) {
        const int64_t cnt = std::min<int64_t>(chunk, num_reads - done);
        a.carry_in = (shared && done > 0) ? 1 : 0;
        B200SA_CUDA(cudaMemsetAsync(plan->qhead.ptr, 0, sizeof(unsigned long long),
                                    plan->stream));
        B200SA_CUDA(cudaEventRecord(plan->ev0, plan->stream));
        rc = launch_items(plan, a, kind_of(plan->hprobs[0]), plan->items_plain.ptr + done, cnt,
                          num_vars, !shared, shared, plan->qhead.ptr, plan->stream, err, errlen,
                          nullptr, plan->hprobs[0].band_w);
        if (rc) return rc;
        B200SA_CUDA(cudaEventRecord(plan->ev1, plan->stream));
        B200SA_CUDA(cudaStreamSynchronize(plan->stream));
        float ms = 0.f;
        B200SA_CUDA(cudaEventElapsedTime(&ms, plan->ev0, plan->ev1));
        total_ms += ms;
        int32_t k = 0;
        for (; k < cnt; ++k) {
            if (interrupt_fn && interrupt_fn(interrupt_ctx)) {  // cpu_sa.cpp:357
                stop = true;
                ++k;
                break;
            }
        }
        // Only completed-and-kept reads are written back; later rows keep
        // their initial states, as in the reference.
        B200SA_CUDA(cudaMemcpyAsync(states + n * (size_t)done, dstates.ptr + n * (size_t)done,
                                    n * (size_t)k, cudaMemcpyDeviceToHost, plan->stream));
        B200SA_CUDA(cudaMemcpyAsync(energies + done, den.ptr + done, sizeof(double) * (size_t)k,
                                    cudaMemcpyDeviceToHost, plan->stream));
        B200SA_CUDA(cudaStreamSynchronize(plan->stream));
        done += k;
    }
    if (stats) {
        rc = collect_stats(plan, {{0, done}}, stats, err, errlen);
        if (rc) return rc;
        stats->kernel_ms = total_ms;
    }
    return done;
}

int b200sa_plan_bucket_report(b200sa_plan plan, b200sa_bucket_report *out, int32_t cap,
                              char *err, size_t errlen) {
    if (!plan) return set_err(err, errlen, B200SA_EINVAL, "plan is NULL");
    if (cap < 0 || (cap > 0 && !out)) return set_err(err, errlen, B200SA_EINVAL, "bad report buffer");
    DeviceGuard guard;
    B200SA_CUDA(cudaSetDevice(plan->device));
    B200SA_CUDA(cudaEventSynchronize(plan->ev1));
    std::vector<ReadStats> hs((size_t)plan->total_reads);
    if (plan->total_reads)
        B200SA_CUDA(cudaMemcpy(hs.data(), plan->dstats.ptr,
                               sizeof(ReadStats) * (size_t)plan->total_reads,
                               cudaMemcpyDeviceToHost));
    int k = 0;
    for (int b = 0; b < kBuckets; ++b) {
        const int64_t o0 = plan->bucket_off[b], o1 = plan->bucket_off[b + 1];
        if (o1 <= o0) continue;
        if (k < cap) {
            b200sa_bucket_report &r = out[k];
            r = b200sa_bucket_report{};
            r.bucket = b;
            r.kind = b % kKinds;
            r.max_n = plan->bucket_max_n[b];
            for (int64_t i = o0; i < o1; ++i) {
                const int64_t it = plan->h_items_lpt[(size_t)i];
                const int p = (int)(it >> 32), rd = (int)(it & 0xffffffffll);
                const ReadStats &x = hs[(size_t)(plan->read_off[p] + rd)];
                const double n = plan->n[p], m = (double)plan->hprobs[p].m;
                const double d = n > 0 ? 2.0 * m / n : 0.0;
                const double att = n * (double)plan->sweeps[p];
                r.reads += 1;
                r.attempts += (int64_t)att;
                r.flips += (int64_t)x.flips;
                r.passes += (int64_t)x.passes;
                // Per read: initial delta energies n(8 + 13d), 9 bytes per
                // attempt, 29d + 9 per flip, final energy 9n + 14m.
                r.model_bytes += n * (8.0 + 13.0 * d) + 9.0 * att +
                                 (double)x.flips * (29.0 * d + 9.0) + 9.0 * n + 14.0 * m;
            }
            r.ms = -1.0;
            if (plan->bucket_timed[b]) {
                float ms = 0.f;
                if (cudaEventElapsedTime(&ms, plan->bev[b][0], plan->bev[b][1]) == cudaSuccess)
                    r.ms = ms;
                else
                    cudaGetLastError();
                const LaunchShape &s = plan->bshape[b];
                r.staging = s.stage;
                r.warps_per_cta = s.warps_per_cta;
                r.grid = s.grid;
                const int rc = variant_reg_class(s.variant);
                r.registers = rc == 1 ? kRegs80 : rc == 2 ? kRegs64 : 128;
            }
        }
        ++k;
    }
    return k;
}

}  // extern "C"
