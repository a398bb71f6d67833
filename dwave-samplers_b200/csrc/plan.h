// Host-side internals of a device-resident plan (b200sa_plan), shared by the
// C ABI (sa_api.cpp) and the launch-graph, weight-update and autotuning code
// (plan_tune.cpp).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <map>
#include <string>
#include <utility>
#include <vector>

#include "b200sa.h"
#include "sa_launch.h"
#include "sa_types.h"

namespace b200sa {
namespace host {

inline int set_err(char *err, size_t errlen, int code, const std::string &msg) {
    if (err && errlen > 0) std::snprintf(err, errlen, "%s", msg.c_str());
    return code;
}

#define B200SA_CUDA(call)                                                        \
    do {                                                                         \
        cudaError_t e_ = (call);                                                 \
        if (e_ != cudaSuccess)                                                   \
            return set_err(err, errlen, B200SA_ECUDA,                            \
                           std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// Restores the caller's current device on scope exit.
struct DeviceGuard {
    int prev = -1;
    DeviceGuard() {
        if (cudaGetDevice(&prev) != cudaSuccess) {
            prev = -1;
            cudaGetLastError();
        }
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};


int select_device(int device, cudaDeviceProp &prop, char *err, size_t errlen);

template <typename T>
struct DevArray {
    T *ptr = nullptr;
    size_t count = 0;
    DevArray() = default;
    DevArray(const DevArray &) = delete;
    DevArray &operator=(const DevArray &) = delete;
    ~DevArray() { release(); }
    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        count = 0;
    }
    cudaError_t alloc(size_t n) {
        release();
        count = n;
        if (n == 0) return cudaSuccess;
        return cudaMalloc(reinterpret_cast<void **>(&ptr), n * sizeof(T));
    }
};

inline size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

// Zeroes the counters of a b200sa_stats, keeping the caller's per-read
// near-tie array pointer (an input).
inline void reset_stats(b200sa_stats *s) {
    if (!s) return;
    uint32_t *keep = s->read_near_ties;
    *s = b200sa_stats{};
    s->read_near_ties = keep;
}

// Nibble tables of the RNG jump by kHalf outputs (computed once per process).
const uint32_t (*jump_table())[4];

// Whether plans enable in-window resolution / dense updates for the problems
// that qualify.
bool resolve_allowed();
bool dense_allowed();
bool band_allowed();

// Buckets of the persistent mode: a size class crossed with the kernel kind
// (acceptance rule x update order).  Each bucket's warps get a shared region
// sized for the bucket's largest n, so small problems pack more resident
// warps per SM; the last size class keeps its state in global memory.
constexpr int kSizeClasses = 8;
constexpr int kGlobalClass = kSizeClasses - 1;
constexpr int kKinds = kNumKinds;
constexpr int kBuckets = kSizeClasses * kKinds;
constexpr int kStreams = 8;
constexpr int kClassBound[kSizeClasses - 2] = {128, 256, 512, 1024, 2048, 4096};

inline int size_class(int n, int onchip_max) {
    if (n > onchip_max) return kGlobalClass;
    for (int b = 0; b < kSizeClasses - 2; ++b)
        if (n <= kClassBound[b]) return b;
    return kSizeClasses - 2;
}

// Kernel kind of a problem: bit 0 Gibbs, bit 1 random order, bit 2
// in-window resolution (sequential order only).
inline int kind_of(const ProblemDev &d) {
    return (d.proposal == 0 ? kKindGibbs : 0) | (d.varorder ? kKindRandom : 0) |
           (d.resolve && !d.varorder ? kKindResolve : 0);
}

// Launch configuration of one bucket chosen by the autotuner (unset: the
// occupancy rule of shape_for).
struct TuneChoice {
    bool set = false;
    int staging = kStageShared;  // state location (kStage*), used where it fits
    int warps_per_cta = 0;
    int ctas_per_sm = 0;    // 0: as many as fit
    int reg_class = 0;      // kernel register budget: 0 = 128, 1 = 80, 2 = 64 per thread
    double rate = 0.0;      // measured attempts/s of the choice
};

struct LaunchShape {
    int stage;         // state location (kStage*)
    int cap_n;         // largest n whose shared-memory part fits the region
    int warps_per_cta;
    int region;
    int grid;
    int variant;
    int touch_bytes;   // random order: the touch bitmap inside the region
    int band_cap;      // kStageBand: slots of the delta-energy band
};

// Arena byte offsets of one packed problem.
struct ArenaOffsets {
    size_t vinfo, dist, share, col, w, h, cu, cv, cw, betas, thr, back, bw, dw, dbits;
};

}  // namespace host
}  // namespace b200sa

struct b200sa_plan_s {
    int device = 0;
    cudaDeviceProp prop{};
    cudaStream_t stream = nullptr;
    cudaStream_t bstream[b200sa::host::kStreams] = {};
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, fork = nullptr;
    cudaEvent_t join[b200sa::host::kStreams] = {};
    int num_problems = 0;
    int onchip_max = 0;
    int onchip_fast = 0;  // untuned: all state on chip up to this n (24 warps' regions per SM)
    std::vector<b200sa::ProblemDev> hprobs;
    std::vector<int32_t> n, reads, sweeps;  // per problem
    std::vector<int64_t> state_off, read_off;
    int64_t total_state = 0, total_reads = 0;
    int32_t max_n = 0;
    b200sa::host::DevArray<uint8_t> arena;
    b200sa::host::DevArray<b200sa::ProblemDev> dprobs;
    b200sa::host::DevArray<uint64_t> dseeds;
    b200sa::host::DevArray<b200sa::ReadStats> dstats;
    b200sa::host::DevArray<int64_t> items_lpt, items_plain;
    b200sa::host::DevArray<unsigned long long> qhead;  // one per bucket
    b200sa::host::DevArray<double> scratch_de;
    b200sa::host::DevArray<int8_t> scratch_s;
    b200sa::host::DevArray<uint64_t> carry;
    int64_t scratch_stride = 0, scratch_slots = 0;
    std::vector<int64_t> plain_item_off;   // per problem offset into items_plain
    int64_t bucket_off[b200sa::host::kBuckets + 1] = {};  // bucket ranges in items_lpt
    int32_t bucket_max_n[b200sa::host::kBuckets] = {};
    // Largest band ring of a bucket whose problems are all banded, else 0.
    int32_t bucket_band_w[b200sa::host::kBuckets] = {};
    int64_t bucket_lead_cost[b200sa::host::kBuckets] = {};
    std::map<std::pair<int, int>, int> occ_cache;  // (variant*2^24 + warps, region) -> CTAs/SM
    int64_t launches = 0;  // sweep-kernel launches issued by the current run
    std::vector<b200sa::host::ArenaOffsets> offs;  // per problem
    std::vector<std::vector<int32_t>> rows;        // per problem: CSR list starts (n + 1)
    std::vector<std::vector<int32_t>> bw_src;      // per problem: adjacency entry of each bw
    // Scatter map of b200sa_plan_set_weights_device (built on first use):
    // arena element sw_dst[i] <- J_cat[sw_src[i]] for i < sw_num_j, else
    // h_cat[sw_src[i]].
    b200sa::host::DevArray<int64_t> sw_dst;
    b200sa::host::DevArray<int32_t> sw_src;
    int64_t sw_num_j = 0, sw_total = -1;
    b200sa::host::TuneChoice tune[b200sa::host::kBuckets];
    // Persistent launches captured as one CUDA graph, valid for the buffers in
    // graph_key (states in, states out, energies, seeds).
    std::vector<int64_t> h_items_lpt;  // host copy of items_lpt
    bool dry_run = false;  // launch_items / run_persistent: shapes and scratch only
    bool capturing = false;  // run_persistent is being captured into the plan's graph
    cudaGraphExec_t graph_exec = nullptr;
    const void *graph_key[4] = {};
    int64_t graph_launches = 0;
    // Timing events around each bucket's launch (recorded on the bucket's
    // stream by persistent runs, and captured into the graph), and the shape
    // of that launch; bucket_timed marks buckets the last such run launched.
    cudaEvent_t bev[b200sa::host::kBuckets][2] = {};
    b200sa::host::LaunchShape bshape[b200sa::host::kBuckets] = {};
    bool bucket_timed[b200sa::host::kBuckets] = {};

    ~b200sa_plan_s() {
        if (graph_exec) cudaGraphExecDestroy(graph_exec);
        for (int b = 0; b < b200sa::host::kBuckets; ++b)
            for (int k = 0; k < 2; ++k)
                if (bev[b][k]) cudaEventDestroy(bev[b][k]);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (fork) cudaEventDestroy(fork);
        for (int b = 0; b < b200sa::host::kStreams; ++b) {
            if (join[b]) cudaEventDestroy(join[b]);
            if (bstream[b]) cudaStreamDestroy(bstream[b]);
        }
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace b200sa {
namespace host {

int occupancy(b200sa_plan_s *P, int variant, int w, int region, int *ctas, char *err,
              size_t errlen);
int shape_for(b200sa_plan_s *P, int kind, int32_t max_n_here, int64_t items, bool persistent,
              LaunchShape &out, char *err, size_t errlen, const TuneChoice *choice = nullptr,
              int band_w_here = 0);
int ensure_scratch(b200sa_plan_s *P, int64_t slots, int64_t stride, char *err, size_t errlen);
LaunchArgs base_args(b200sa_plan_s *P, const int8_t *in, int8_t *out, double *en,
                     const uint64_t *seeds);
int launch_items(b200sa_plan_s *P, LaunchArgs a, int kind, const int64_t *items, int64_t count,
                 int32_t max_n_here, bool persistent, bool shared_stream,
                 unsigned long long *qhead, cudaStream_t st, char *err, size_t errlen,
                 const TuneChoice *choice = nullptr, int band_w_here = 0);
int collect_stats(b200sa_plan_s *P, const std::vector<std::pair<int, int>> &ranges,
                  b200sa_stats *stats, char *err, size_t errlen);
int run_persistent(b200sa_plan_s *P, LaunchArgs a, cudaStream_t st, char *err, size_t errlen);
// B200SA_MODE_GRAPH: captures run_persistent once per buffer set, then replays.
int run_graph(b200sa_plan_s *P, LaunchArgs a, cudaStream_t st, char *err, size_t errlen);

}  // namespace host
}  // namespace b200sa
