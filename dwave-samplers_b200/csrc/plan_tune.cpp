// Plan extensions with no reference counterpart: the persistent launches
// captured as a CUDA graph, in-place weight updates for learning loops, and
// the measured launch-configuration autotuner with its on-disk cache.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "plan.h"

using namespace b200sa;
using namespace b200sa::host;

namespace b200sa {
namespace host {

// Shapes (and global scratch) of every bucket are settled by a dry pass
// before the capture, so nothing is allocated or queried while capturing.
int run_graph(b200sa_plan_s *P, LaunchArgs a, cudaStream_t st, char *err, size_t errlen) {
    const void *key[4] = {a.states_in, a.states_out, a.energies, a.seeds};
    if (!P->graph_exec || std::memcmp(key, P->graph_key, sizeof(key)) != 0) {
        if (P->graph_exec) {
            B200SA_CUDA(cudaStreamSynchronize(st));
            cudaGraphExecDestroy(P->graph_exec);
            P->graph_exec = nullptr;
        }
        P->dry_run = true;
        int rc = run_persistent(P, a, P->stream, err, errlen);
        P->dry_run = false;
        if (rc) return rc;
        B200SA_CUDA(cudaStreamSynchronize(P->stream));
        B200SA_CUDA(cudaStreamBeginCapture(P->stream, cudaStreamCaptureModeRelaxed));
        P->launches = 0;
        P->capturing = true;
        rc = run_persistent(P, a, P->stream, err, errlen);
        P->capturing = false;
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(P->stream, &g);
        if (rc) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        B200SA_CUDA(e);
        const cudaError_t ei = cudaGraphInstantiate(&P->graph_exec, g, 0);
        cudaGraphDestroy(g);
        if (ei != cudaSuccess) P->graph_exec = nullptr;
        B200SA_CUDA(ei);
        std::memcpy(P->graph_key, key, sizeof(key));
        P->graph_launches = P->launches;
    }
    B200SA_CUDA(cudaGraphLaunch(P->graph_exec, st));
    P->launches = P->graph_launches;
    return B200SA_OK;
}

namespace {

// ---- autotuner ---------------------------------------------------------------

constexpr int kTuneBetas = 8;     // betas per sampled schedule
constexpr int kTuneWarpsPerSm = 64;  // sample reads per SM: two waves at 32 warps per SM

std::string tune_key(const b200sa_plan_s *P, int kind, int max_n, int mean_degree) {
    std::string name = P->prop.name;
    for (char &c : name)
        if (c == ' ' || c == ';' || c == '=') c = '_';
    const int n_bin = (max_n + 63) / 64 * 64;
    std::ostringstream k;
    k << "gpu=" << name << ";sms=" << P->prop.multiProcessorCount << ";lib=" << b200sa_version()
      << ";kind=" << kind << ";n=" << n_bin << ";deg=" << mean_degree;
    std::string s = k.str();
    for (char &c : s)
        if (c == ' ') c = '_';
    return s;
}

// Cache lines: "<key> <staging> <warps_per_cta> <ctas_per_sm> <reg_class> <attempts/s>".
std::map<std::string, TuneChoice> load_cache(const char *path) {
    std::map<std::string, TuneChoice> out;
    if (!path) return out;
    std::ifstream f(path);
    std::string line;
    while (std::getline(f, line)) {
        std::istringstream in(line);
        std::string key;
        int staging = 0, w = 0, ctas = 0, regs = 0;
        double rate = 0.0;
        if (!(in >> key >> staging >> w >> ctas >> regs >> rate)) continue;
        if (w < 1 || w > kMaxThreadsPerCta / 32 || ctas < 0 || regs < 0 || regs >= kRegClasses ||
            staging < kStageGlobal || staging > kStageBand)
            continue;
        TuneChoice c;
        c.set = true;
        c.staging = staging;
        c.warps_per_cta = w;
        c.ctas_per_sm = ctas;
        c.reg_class = regs;
        c.rate = rate;
        out[key] = c;
    }
    return out;
}

bool save_cache(const char *path, const std::map<std::string, TuneChoice> &cache) {
    if (!path) return true;
    const std::string tmp = std::string(path) + ".tmp";
    {
        std::ofstream f(tmp, std::ios::trunc);
        if (!f) return false;
        for (const auto &kv : cache)
            f << kv.first << ' ' << kv.second.staging << ' ' << kv.second.warps_per_cta
              << ' ' << kv.second.ctas_per_sm << ' ' << kv.second.reg_class << ' '
              << kv.second.rate << '\n';
        if (!f) return false;
    }
    return std::rename(tmp.c_str(), path) == 0;
}

// The sample a bucket is timed on: its first (largest, in LPT order) items,
// each problem's schedule cut to kTuneBetas betas spread over it with one
// sweep each, states and outputs in buffers of their own.
struct TuneSample {
    DevArray<ProblemDev> probs;
    DevArray<int64_t> items;
    DevArray<double> sched;  // betas then thresholds, kTuneBetas per problem
    DevArray<int8_t> states_in, states_out;
    DevArray<double> energies;
    DevArray<uint64_t> seeds;
    DevArray<ReadStats> stats;
    DevArray<unsigned long long> qhead;
    int64_t count = 0;
    double attempts = 0.0;
};

int build_sample(b200sa_plan_s *P, int b, int64_t max_items, TuneSample &S, int *mean_degree,
                 char *err, size_t errlen) {
    const int64_t off = P->bucket_off[b];
    const int64_t cnt = std::min<int64_t>(P->bucket_off[b + 1] - off, max_items);
    std::map<int, int> local;  // plan problem -> sample problem
    std::vector<ProblemDev> probs;
    std::vector<int64_t> items;
    std::vector<int32_t> reads;
    for (int64_t i = 0; i < cnt; ++i) {
        const int64_t it = P->h_items_lpt[(size_t)(off + i)];
        const int p = (int)(it >> 32);
        auto f = local.find(p);
        int lp;
        if (f == local.end()) {
            lp = (int)probs.size();
            local[p] = lp;
            probs.push_back(P->hprobs[p]);
            reads.push_back(0);
        } else {
            lp = f->second;
        }
        items.push_back(((int64_t)lp << 32) | reads[lp]);
        reads[lp]++;
    }
    const int np = (int)probs.size();
    std::vector<double> sched((size_t)np * 2 * kTuneBetas);
    // Each sampled schedule: kTuneBetas betas at the midpoints of equal
    // parts of the problem's schedule (read back from the plan's arena).
    int64_t state_total = 0, read_total = 0, vars = 0, entries = 0;
    for (int lp = 0; lp < np; ++lp) {
        ProblemDev &d = probs[lp];
        const int nb = d.num_betas;
        std::vector<double> betas((size_t)std::max(nb, 1));
        if (nb > 0)
            B200SA_CUDA(cudaMemcpy(betas.data(), d.betas, sizeof(double) * (size_t)nb,
                                   cudaMemcpyDeviceToHost));
        const int t = std::min(nb, kTuneBetas);
        for (int j = 0; j < t; ++j) {
            const double beta = betas[(size_t)(((int64_t)j * 2 + 1) * nb / (2 * t))];
            sched[(size_t)lp * 2 * kTuneBetas + j] = beta;
            sched[(size_t)lp * 2 * kTuneBetas + kTuneBetas + j] = 44.36142 / beta;
        }
        d.num_betas = t;
        d.sweeps_per_beta = 1;
        d.num_reads = reads[lp];
        d.state_offset = state_total;
        d.read_offset = read_total;
        state_total += (int64_t)reads[lp] * d.n;
        read_total += reads[lp];
        S.attempts += (double)reads[lp] * (double)d.n * t;
        vars += d.n;
        entries += 2 * d.m;
    }
    *mean_degree = vars > 0 ? (int)std::lround((double)entries / (double)vars) : 0;
    B200SA_CUDA(S.sched.alloc(sched.size()));
    for (int lp = 0; lp < np; ++lp) {
        probs[lp].betas = S.sched.ptr + (size_t)lp * 2 * kTuneBetas;
        probs[lp].thresholds = S.sched.ptr + (size_t)lp * 2 * kTuneBetas + kTuneBetas;
    }
    std::vector<int8_t> st((size_t)std::max<int64_t>(state_total, 1));
    uint64_t x = 0x9E3779B97F4A7C15ull;
    for (auto &v : st) {  // uniform +-1 initial states (xorshift64)
        x ^= x << 13;
        x ^= x >> 7;
        x ^= x << 17;
        v = (x >> 63) ? 1 : -1;
    }
    std::vector<uint64_t> seeds((size_t)std::max<int64_t>(read_total, 1));
    for (size_t i = 0; i < seeds.size(); ++i) seeds[i] = 1 + i;
    B200SA_CUDA(S.probs.alloc((size_t)std::max(np, 1)));
    B200SA_CUDA(S.items.alloc((size_t)std::max<int64_t>(cnt, 1)));
    B200SA_CUDA(S.states_in.alloc(st.size()));
    B200SA_CUDA(S.states_out.alloc(st.size()));
    B200SA_CUDA(S.energies.alloc(seeds.size()));
    B200SA_CUDA(S.seeds.alloc(seeds.size()));
    B200SA_CUDA(S.stats.alloc(seeds.size()));
    B200SA_CUDA(S.qhead.alloc(1));
    if (np)
        B200SA_CUDA(cudaMemcpy(S.probs.ptr, probs.data(), sizeof(ProblemDev) * (size_t)np,
                               cudaMemcpyHostToDevice));
    if (cnt)
        B200SA_CUDA(cudaMemcpy(S.items.ptr, items.data(), 8 * (size_t)cnt, cudaMemcpyHostToDevice));
    B200SA_CUDA(cudaMemcpy(S.sched.ptr, sched.data(), 8 * sched.size(), cudaMemcpyHostToDevice));
    B200SA_CUDA(cudaMemcpy(S.states_in.ptr, st.data(), st.size(), cudaMemcpyHostToDevice));
    B200SA_CUDA(cudaMemcpy(S.seeds.ptr, seeds.data(), 8 * seeds.size(), cudaMemcpyHostToDevice));
    S.count = cnt;
    return B200SA_OK;
}

// Best of two timed launches of one candidate on the sample (ms).
int time_candidate(b200sa_plan_s *P, int kind, int max_n, int band_w, const TuneChoice &c,
                   TuneSample &S, float *best_ms, char *err, size_t errlen) {
    LaunchShape s{};
    int rc = shape_for(P, kind, max_n, S.count, true, s, err, errlen, &c, band_w);
    if (rc) return rc;
    if (s.stage != kStageShared) {
        rc = ensure_scratch(P, (int64_t)s.grid * s.warps_per_cta, max_n, err, errlen);
        if (rc) return rc;
    }
    LaunchArgs a{};
    a.problems = S.probs.ptr;
    a.states_in = S.states_in.ptr;
    a.states_out = S.states_out.ptr;
    a.energies = S.energies.ptr;
    a.seeds = S.seeds.ptr;
    a.stats = S.stats.ptr;
    a.items = S.items.ptr;
    a.num_items = S.count;
    a.smem_cap_n = s.cap_n;
    a.touch_bytes = s.touch_bytes;
    a.band_cap = s.band_cap;
    a.scratch_de = P->scratch_de.ptr;
    a.scratch_s = P->scratch_s.ptr;
    a.scratch_stride = P->scratch_stride;
    a.num_slots = P->scratch_slots;
    a.queue_head = S.qhead.ptr;
    *best_ms = 0.f;
    for (int rep = 0; rep < 2; ++rep) {
        B200SA_CUDA(cudaMemsetAsync(S.qhead.ptr, 0, sizeof(unsigned long long), P->stream));
        B200SA_CUDA(cudaEventRecord(P->ev0, P->stream));
        B200SA_CUDA(launch_sa(s.variant, a, s.grid, s.warps_per_cta, s.region, P->stream));
        B200SA_CUDA(cudaEventRecord(P->ev1, P->stream));
        B200SA_CUDA(cudaStreamSynchronize(P->stream));
        float ms = 0.f;
        B200SA_CUDA(cudaEventElapsedTime(&ms, P->ev0, P->ev1));
        if (rep == 0 || ms < *best_ms) *best_ms = ms;
    }
    return B200SA_OK;
}

}  // namespace
}  // namespace host
}  // namespace b200sa

extern "C" {

int b200sa_plan_set_weights(b200sa_plan plan, int32_t problem, const double *h, const double *J,
                            char *err, size_t errlen) {
    if (!plan) return set_err(err, errlen, B200SA_EINVAL, "plan is NULL");
    if (problem < 0 || problem >= plan->num_problems)
        return set_err(err, errlen, B200SA_EINVAL, "problem index out of range");
    const ProblemDev &d = plan->hprobs[problem];
    const int n = d.n;
    const int64_t m = d.m;
    if ((n > 0 && !h) || (m > 0 && !J))
        return set_err(err, errlen, B200SA_EINVAL, "h or J is NULL");
    DeviceGuard guard;
    B200SA_CUDA(cudaSetDevice(plan->device));
    // Coupler c's weight goes to the list positions the packer gave it: the
    // lists are filled in coupler order (cpu_sa.cpp:298-316), so replaying
    // that fill with the same list starts lands every weight in place.
    const std::vector<int32_t> &row = plan->rows[problem];
    std::vector<int32_t> hcu((size_t)m), hcv((size_t)m);
    std::vector<double> w((size_t)(2 * m));
    if (m) {
        B200SA_CUDA(cudaMemcpy(hcu.data(), d.cu, 4 * (size_t)m, cudaMemcpyDeviceToHost));
        B200SA_CUDA(cudaMemcpy(hcv.data(), d.cv, 4 * (size_t)m, cudaMemcpyDeviceToHost));
        std::vector<int32_t> cur(row.begin(), row.end() - 1);
        for (int64_t c = 0; c < m; ++c) {
            w[(size_t)cur[hcu[c]]++] = J[c];
            w[(size_t)cur[hcv[c]]++] = J[c];
        }
    }
    const ArenaOffsets &o = plan->offs[problem];
    uint8_t *base = plan->arena.ptr;
    // After the plan's last run (its end event) on the plan's own stream.
    B200SA_CUDA(cudaStreamWaitEvent(plan->stream, plan->ev1, 0));
    if (n) B200SA_CUDA(cudaMemcpyAsync(base + o.h, h, 8 * (size_t)n, cudaMemcpyHostToDevice,
                                       plan->stream));
    // The back-neighbour couplings of the in-window resolution are copies of
    // adjacency entries.
    const std::vector<int32_t> &src = plan->bw_src[problem];
    std::vector<double> bw(src.size());
    for (size_t i = 0; i < src.size(); ++i) bw[i] = w[(size_t)src[i]];
    if (m) {
        B200SA_CUDA(cudaMemcpyAsync(base + o.w, w.data(), 8 * (size_t)(2 * m),
                                    cudaMemcpyHostToDevice, plan->stream));
        B200SA_CUDA(cudaMemcpyAsync(base + o.cw, J, 8 * (size_t)m, cudaMemcpyHostToDevice,
                                    plan->stream));
    }
    if (!bw.empty())
        B200SA_CUDA(cudaMemcpyAsync(base + o.bw, bw.data(), 8 * bw.size(),
                                    cudaMemcpyHostToDevice, plan->stream));
    // The dense coupling matrix of problems with dense updates (no repeated
    // couplers there, so each entry is one coupler's weight).
    std::vector<double> dw;
    if (d.dense) {
        dw.assign((size_t)n * (size_t)n, 0.0);
        for (int64_t c = 0; c < m; ++c) {
            dw[(size_t)hcu[c] * n + hcv[c]] = J[c];
            dw[(size_t)hcv[c] * n + hcu[c]] = J[c];
        }
        B200SA_CUDA(cudaMemcpyAsync(base + o.dw, dw.data(), 8 * dw.size(),
                                    cudaMemcpyHostToDevice, plan->stream));
    }
    B200SA_CUDA(cudaStreamSynchronize(plan->stream));
    return B200SA_OK;
}

int b200sa_plan_set_weights_device(b200sa_plan plan, const double *d_h, const double *d_J,
                                   void *stream, char *err, size_t errlen) {
    if (!plan) return set_err(err, errlen, B200SA_EINVAL, "plan is NULL");
    int64_t total_n = 0, total_m = 0;
    for (int i = 0; i < plan->num_problems; ++i) {
        total_n += plan->hprobs[i].n;
        total_m += plan->hprobs[i].m;
    }
    if ((total_n > 0 && !d_h) || (total_m > 0 && !d_J))
        return set_err(err, errlen, B200SA_EINVAL, "h or J is NULL");
    if (total_n + total_m > (int64_t)INT32_MAX)
        return set_err(err, errlen, B200SA_EINVAL, "too many fields and couplers");
    DeviceGuard guard;
    B200SA_CUDA(cudaSetDevice(plan->device));
    if (plan->sw_total < 0) {
        // Each coupler's weight goes to its two adjacency entries (the
        // packer's fill order, cpu_sa.cpp:298-316, replayed from the list
        // starts), to its COO copy and to the back-neighbour copies of those
        // entries; each field to its slot.
        std::vector<int64_t> dst;
        std::vector<int32_t> src;
        std::vector<int64_t> hdst;
        std::vector<int32_t> hsrc;
        int64_t joff = 0, hoff = 0;
        for (int i = 0; i < plan->num_problems; ++i) {
            const ProblemDev &d = plan->hprobs[i];
            const ArenaOffsets &o = plan->offs[i];
            const int64_t m = d.m;
            std::vector<int32_t> hcu((size_t)m), hcv((size_t)m), coupler((size_t)(2 * m));
            if (m) {
                B200SA_CUDA(cudaMemcpy(hcu.data(), d.cu, 4 * (size_t)m, cudaMemcpyDeviceToHost));
                B200SA_CUDA(cudaMemcpy(hcv.data(), d.cv, 4 * (size_t)m, cudaMemcpyDeviceToHost));
            }
            const std::vector<int32_t> &row = plan->rows[i];
            std::vector<int32_t> cur(row.begin(), row.end() - 1);
            for (int64_t c = 0; c < m; ++c) {
                const int32_t eu = cur[hcu[c]]++, ev = cur[hcv[c]]++;
                coupler[(size_t)eu] = (int32_t)c;
                coupler[(size_t)ev] = (int32_t)c;
                dst.push_back((int64_t)(o.w / 8) + eu);
                src.push_back((int32_t)(joff + c));
                dst.push_back((int64_t)(o.w / 8) + ev);
                src.push_back((int32_t)(joff + c));
                dst.push_back((int64_t)(o.cw / 8) + c);
                src.push_back((int32_t)(joff + c));
                if (d.dense) {  // the dense coupling matrix, both triangles
                    dst.push_back((int64_t)(o.dw / 8) + (int64_t)hcu[c] * d.n + hcv[c]);
                    src.push_back((int32_t)(joff + c));
                    dst.push_back((int64_t)(o.dw / 8) + (int64_t)hcv[c] * d.n + hcu[c]);
                    src.push_back((int32_t)(joff + c));
                }
            }
            const std::vector<int32_t> &bs = plan->bw_src[i];
            for (size_t k = 0; k < bs.size(); ++k) {
                dst.push_back((int64_t)(o.bw / 8) + (int64_t)k);
                src.push_back((int32_t)(joff + coupler[(size_t)bs[k]]));
            }
            for (int32_t v = 0; v < d.n; ++v) {
                hdst.push_back((int64_t)(o.h / 8) + v);
                hsrc.push_back((int32_t)(hoff + v));
            }
            joff += m;
            hoff += d.n;
        }
        const int64_t num_j = (int64_t)dst.size();
        dst.insert(dst.end(), hdst.begin(), hdst.end());
        src.insert(src.end(), hsrc.begin(), hsrc.end());
        B200SA_CUDA(plan->sw_dst.alloc(std::max<size_t>(dst.size(), 1)));
        B200SA_CUDA(plan->sw_src.alloc(std::max<size_t>(src.size(), 1)));
        if (!dst.empty()) {
            B200SA_CUDA(cudaMemcpy(plan->sw_dst.ptr, dst.data(), 8 * dst.size(),
                                   cudaMemcpyHostToDevice));
            B200SA_CUDA(cudaMemcpy(plan->sw_src.ptr, src.data(), 4 * src.size(),
                                   cudaMemcpyHostToDevice));
        }
        plan->sw_num_j = num_j;
        plan->sw_total = (int64_t)dst.size();
    }
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : plan->stream;
    B200SA_CUDA(scatter_weights(reinterpret_cast<double *>(plan->arena.ptr), plan->sw_dst.ptr,
                                plan->sw_src.ptr, plan->sw_num_j, plan->sw_total, d_J, d_h, st));
    return B200SA_OK;
}

int b200sa_plan_autotune(b200sa_plan plan, const char *cache_path, int32_t flags,
                         b200sa_tune_entry *report, int32_t report_cap, char *err,
                         size_t errlen) {
    if (!plan) return set_err(err, errlen, B200SA_EINVAL, "plan is NULL");
    if (report_cap < 0 || (report_cap > 0 && !report))
        return set_err(err, errlen, B200SA_EINVAL, "bad report buffer");
    DeviceGuard guard;
    B200SA_CUDA(cudaSetDevice(plan->device));
    B200SA_CUDA(cudaDeviceSynchronize());
    std::map<std::string, TuneChoice> cache = load_cache(cache_path);
    const int sms = plan->prop.multiProcessorCount;
    const int smem_blk = (int)plan->prop.sharedMemPerBlockOptin;
    int buckets = 0;
    bool changed = false;
    for (int b = 0; b < kBuckets; ++b) {
        const int64_t cnt = plan->bucket_off[b + 1] - plan->bucket_off[b];
        if (cnt <= 0) continue;
        const int kind = b % kKinds;
        const int max_n = plan->bucket_max_n[b];
        const int band_w = plan->bucket_band_w[b];
        TuneSample S;
        int mean_degree = 0;
        int rc = build_sample(plan, b, (int64_t)sms * kTuneWarpsPerSm, S, &mean_degree,
                              err, errlen);
        if (rc) return rc;
        const std::string key = tune_key(plan, kind, max_n, mean_degree);
        TuneChoice best;
        int measured = 0;
        bool cached = false;
        auto hit = cache.find(key);
        if (!(flags & B200SA_TUNE_FORCE) && hit != cache.end()) {
            best = hit->second;
            cached = true;
        } else {
            // Candidates: per register budget and staging, every
            // warps-per-CTA whose resident warps per SM come within 7/8 of
            // that pair's best, at full occupancy, plus the largest such CTA
            // with one CTA fewer per SM (more L1 beside the shared regions).
            std::vector<TuneChoice> cands;
            for (int regs = 0; regs < kRegClasses; ++regs)
            for (int stage : {kStageShared, kStageSpins, kStageGlobal, kStageBand}) {
                if (stage == kStageShared && max_n > plan->onchip_max) continue;
                if (stage == kStageBand && (!band_w || (kind & kKindRandom))) continue;
                const int region =
                    region_bytes_for_stage(stage, stage == kStageGlobal ? 0 : max_n,
                                           stage == kStageBand ? band_w : 0) +
                    touch_bytes_for((kind & kKindRandom) != 0, max_n);
                if (region > smem_blk) continue;
                const int variant = kernel_variant(kind, stage, regs);
                int resident[kMaxThreadsPerCta / 32 + 1] = {};
                int ctas_of[kMaxThreadsPerCta / 32 + 1] = {};
                int top = 0;
                for (int w = 1; w <= kMaxThreadsPerCta / 32; ++w) {
                    if ((int64_t)w * region > smem_blk) break;
                    rc = occupancy(plan, variant, w, region, &ctas_of[w], err, errlen);
                    if (rc) return rc;
                    resident[w] = ctas_of[w] * w;
                    top = std::max(top, resident[w]);
                }
                int widest = 0;
                for (int w = 1; w <= kMaxThreadsPerCta / 32; ++w) {
                    if (resident[w] == 0 || 8 * resident[w] < 7 * top) continue;
                    TuneChoice c;
                    c.set = true;
                    c.staging = stage;
                    c.warps_per_cta = w;
                    c.reg_class = regs;
                    cands.push_back(c);
                    widest = w;
                }
                if (widest && ctas_of[widest] > 1) {
                    TuneChoice c = cands.back();
                    c.ctas_per_sm = ctas_of[widest] - 1;
                    cands.push_back(c);
                }
                // State in global slots: fewer resident warps also means
                // fewer slots competing for L2 (delta energies, 8 bytes a
                // variable, and spins for the global location).  Offer the
                // widest CTA with its CTAs per SM capped so that the slots
                // fit in 40% and in 70% of L2.
                if (widest && (stage == kStageGlobal || stage == kStageSpins)) {
                    const double per_warp = (double)max_n * (stage == kStageGlobal ? 9.0 : 8.0);
                    const double l2 = (double)plan->prop.l2CacheSize;
                    int last_cap = ctas_of[widest] - 1;
                    for (double share : {0.7, 0.4}) {
                        const int cap = (int)(share * l2 / (per_warp * sms * widest));
                        if (cap < 1 || cap >= last_cap) continue;
                        TuneChoice c;
                        c.set = true;
                        c.staging = stage;
                        c.warps_per_cta = widest;
                        c.reg_class = regs;
                        c.ctas_per_sm = cap;
                        cands.push_back(c);
                        last_cap = cap;
                    }
                }
            }
            float best_ms = 0.f;
            // B200SA_TUNE_LOG names a file that receives one line per measured
            // candidate (the evidence behind each choice).
            const char *log_path = std::getenv("B200SA_TUNE_LOG");
            std::ofstream tlog;
            if (log_path && *log_path) tlog.open(log_path, std::ios::app);
            for (const TuneChoice &c : cands) {
                float ms = 0.f;
                rc = time_candidate(plan, kind, max_n, band_w, c, S, &ms, err, errlen);
                if (rc) return rc;
                ++measured;
                if (tlog)
                    tlog << "kind=" << kind << " max_n=" << max_n << " items=" << S.count
                         << " staging=" << c.staging << " warps_per_cta=" << c.warps_per_cta
                         << " ctas_per_sm=" << c.ctas_per_sm << " registers="
                         << (c.reg_class == 1 ? kRegs80 : c.reg_class == 2 ? kRegs64 : 128)
                         << " ms=" << ms << " attempts_per_s="
                         << (ms > 0.f ? S.attempts / (ms * 1e-3) : 0.0) << '\n';
                if (!best.set || ms < best_ms) {
                    best = c;
                    best_ms = ms;
                    best.rate = ms > 0.f ? S.attempts / (ms * 1e-3) : 0.0;
                }
            }
            if (best.set) {
                cache[key] = best;
                changed = true;
            }
        }
        plan->tune[b] = best;
        if (buckets < report_cap) {
            b200sa_tune_entry &e = report[buckets];
            e.bucket = b;
            e.kind = kind;
            e.max_n = max_n;
            e.items = cnt;
            e.staging = best.staging;
            e.warps_per_cta = best.warps_per_cta;
            e.ctas_per_sm = best.ctas_per_sm;
            e.registers = best.reg_class == 1 ? kRegs80 : best.reg_class == 2 ? kRegs64 : 128;
            e.attempts_per_s = best.rate;
            e.from_cache = cached ? 1 : 0;
            e.candidates = measured;
        }
        ++buckets;
    }
    // A captured graph holds the old shapes.
    if (plan->graph_exec) {
        cudaGraphExecDestroy(plan->graph_exec);
        plan->graph_exec = nullptr;
    }
    if (changed && !save_cache(cache_path, cache))
        return set_err(err, errlen, B200SA_EINVAL,
                       std::string("cannot write the tuning cache ") + cache_path);
    return buckets;
}

}  // extern "C"
