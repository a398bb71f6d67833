// b200sa_sample_noalloc: the sampler without any memory allocation.
//
// Some callers cannot allocate device memory while they run: code that owns
// all device memory through a pre-sized pool or arena and forbids further
// allocations, plugin hosts that only allow allocations at start-up, and
// latency-critical loops where cudaMalloc / cudaFree (which may synchronize
// the whole device) are not acceptable.  This entry point takes every input
// and output as device memory the caller already owns, and keeps all of its
// own working memory in one fixed array that is part of the loaded library
// (`g_noalloc_scratch`, kNoAllocScratchBytes bytes per device, held until the
// process exits).  It allocates nothing on the device or on the host heap.
//
// That working memory bounds the problem size (see the kNoAllocMax*
// constants); larger problems are rejected with B200SA_EINVAL.  Every call on
// a device reuses the same array and leaves its contents behind; each call
// clears what it needs at zero itself.  Calls that overlap on the GPU (two
// host threads, or two streams, on the same device at once) race on the array
// and must be serialized by the caller.
//
// The first call on each device resolves the array's device address with
// cudaGetSymbolAddress, uploads the RNG jump table and reads the device's
// properties once.  Every call waits for its own work (it reads an error flag
// and the near-tie total back to the host), so a call cannot be recorded
// into a CUDA graph: a call made while its stream is capturing returns
// B200SA_EINVAL before doing anything.
//
// The annealing itself is the regular sweep kernel, unchanged; only its
// inputs (packed adjacency, thresholds, work items, counters) are prepared
// on the device inside the fixed array instead of in allocated buffers.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "b200sa.h"
#include "pack.h"
#include "sa_launch.h"
#include "sa_types.h"

namespace b200sa {
namespace {

constexpr int64_t kNoAllocMaxVars = 4096;
constexpr int64_t kNoAllocMaxCouplers = 65536;
constexpr int64_t kNoAllocMaxBetas = 16384;
constexpr int64_t kNoAllocMaxReads = 16384;

constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Byte offsets of the working areas inside the fixed array.
constexpr size_t kOffErr = 0;                                      // int error flag
constexpr size_t kOffTies = 64;                                    // near-tie total (u64)
constexpr size_t kOffQueue = 256;                                  // work-queue head
constexpr size_t kOffProb = 512;                                   // ProblemDev
constexpr size_t kOffCursor = align256(kOffProb + sizeof(ProblemDev));  // int[n]
constexpr size_t kOffVinfo = align256(kOffCursor + 4 * kNoAllocMaxVars);
constexpr size_t kOffDist = align256(kOffVinfo + 8 * kNoAllocMaxVars);
constexpr size_t kOffShare = align256(kOffDist + kNoAllocMaxVars);
constexpr size_t kOffCol = align256(kOffShare + 4 * kNoAllocMaxVars);
constexpr size_t kOffW = align256(kOffCol + 4 * 2 * kNoAllocMaxCouplers);
constexpr size_t kOffThr = align256(kOffW + 8 * 2 * kNoAllocMaxCouplers);
constexpr size_t kOffItems = align256(kOffThr + 8 * kNoAllocMaxBetas);
constexpr size_t kOffStats = align256(kOffItems + 8 * kNoAllocMaxReads);
constexpr size_t kUsed = align256(kOffStats + sizeof(ReadStats) * kNoAllocMaxReads);
constexpr size_t kNoAllocScratchBytes = size_t(4) << 20;  // 4 MiB
static_assert(kUsed <= kNoAllocScratchBytes, "working areas exceed the fixed array");

// The library's fixed working memory.  Host code must not pass this name to
// a kernel (on the host it is only a stand-in); it passes the address that
// cudaGetSymbolAddress returns.  Device code in this file may name it.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

struct PackArgs {
    unsigned char *base;  // device address of g_noalloc_scratch
    int n;
    int64_t m;
    const double *h;
    const int32_t *cu;
    const int32_t *cv;
    const double *cw;
    int num_betas;
    const double *betas;
    int num_reads;
    int sweeps_per_beta;
    int varorder;
    int proposal;
};

// Builds the order-preserving adjacency (cpu_sa.cpp:298-316), the
// per-variable records, the skip thresholds (cpu_sa.cpp:131) and the work
// items inside the fixed array.  One block; out-of-range coupler indices set
// the error flag and nothing is built.
__global__ void __launch_bounds__(1024) noalloc_pack_kernel(PackArgs a) {
    __shared__ int s_err;
    __shared__ int s_cursor[kNoAllocMaxVars];  // next free position of each list
    __shared__ int s_tgt[64];                  // the targets of one chunk's 64 entries
    int *err = reinterpret_cast<int *>(a.base + kOffErr);
    unsigned long long *queue = reinterpret_cast<unsigned long long *>(a.base + kOffQueue);
    int *cursor = reinterpret_cast<int *>(a.base + kOffCursor);
    uint2 *vinfo = reinterpret_cast<uint2 *>(a.base + kOffVinfo);
    uint8_t *dist = a.base + kOffDist;
    uint32_t *share = reinterpret_cast<uint32_t *>(a.base + kOffShare);
    int32_t *col = reinterpret_cast<int32_t *>(a.base + kOffCol);
    double *w = reinterpret_cast<double *>(a.base + kOffW);
    double *thr = reinterpret_cast<double *>(a.base + kOffThr);
    int64_t *items = reinterpret_cast<int64_t *>(a.base + kOffItems);
    const int tid = threadIdx.x, nt = blockDim.x;

    // What must start at zero: the error flag, the queue head, the degrees.
    if (tid == 0) {
        s_err = 0;
        *err = 0;
        *queue = 0ull;
    }
    for (int v = tid; v < a.n; v += nt) cursor[v] = 0;
    __syncthreads();
    for (int64_t c = tid; c < a.m; c += nt) {
        const int u = a.cu[c], v = a.cv[c];
        if (u < 0 || v < 0 || u >= a.n || v >= a.n) {
            atomicExch(&s_err, 1);
        } else {
            atomicAdd(&cursor[u], 1);
            atomicAdd(&cursor[v], 1);
        }
    }
    __syncthreads();
    if (s_err) {
        if (tid == 0) *err = 1;
        return;
    }
    // Degrees -> list starts (exclusive scan; n <= 4096, one thread).
    if (tid == 0) {
        int run = 0;
        for (int v = 0; v < a.n; ++v) {
            const int d = cursor[v];
            vinfo[v] = make_uint2((unsigned)run, (unsigned)d);
            s_cursor[v] = run;
            run += d;
        }
    }
    __syncthreads();
    // Fill in coupler order (each list keeps the input order, cpu_sa.cpp:
    // 298-316), one warp, 32 couplers at a time: coupler c pushes u's entry,
    // then v's; an entry's position is its list's cursor plus the entries of
    // earlier couplers of the chunk (and, for v's entry of a self-loop, u's)
    // that name the same list.
    if (tid < 32) {
        for (int64_t base = 0; base < a.m; base += 32) {
            const int64_t c = base + tid;
            const bool ok = c < a.m;
            int u = -1, v = -2;
            double J = 0.0;
            if (ok) {
                u = a.cu[c];
                v = a.cv[c];
                J = a.cw[c];
            }
            s_tgt[2 * tid] = ok ? u : -1;
            s_tgt[2 * tid + 1] = ok ? v : -2;
            __syncwarp();
            if (ok) {
                int ru = 0, rv = (u == v) ? 1 : 0;
                for (int j = 0; j < 2 * tid; ++j) {
                    const int t = s_tgt[j];
                    ru += t == u;
                    rv += t == v;
                }
                const int ku = s_cursor[u] + ru, kv = s_cursor[v] + rv;
                col[ku] = v;
                w[ku] = J;
                col[kv] = u;
                w[kv] = J;
            }
            __syncwarp();
            if (ok) {  // the chunk's counts; every lane has read the cursors
                atomicAdd(&s_cursor[u], 1);
                atomicAdd(&s_cursor[v], 1);
            }
            __syncwarp();
        }
    }
    __syncthreads();
    // Speculation records: nearest later neighbour; conflict masks set
    // conservatively (all bits) so the sweep always groups equal targets.
    for (int v = tid; v < a.n; v += nt) {
        const uint2 vi = vinfo[v];
        unsigned dmin = kDistCap;
        for (unsigned e = vi.x; e < vi.x + vi.y; ++e) {
            const int u = col[e];
            if (u > v && (unsigned)(u - v) < dmin) dmin = (unsigned)(u - v);
        }
        dist[v] = (uint8_t)dmin;
        share[v] = ~0u;
    }
    for (int b = tid; b < a.num_betas; b += nt) thr[b] = 44.36142 / a.betas[b];
    for (int r = tid; r < a.num_reads; r += nt) items[r] = (int64_t)r;  // problem 0, read r
    if (tid == 0) {
        ProblemDev *P = reinterpret_cast<ProblemDev *>(a.base + kOffProb);
        P->n = a.n;
        P->sweeps_per_beta = a.sweeps_per_beta;
        P->num_betas = a.num_betas;
        P->num_reads = a.num_reads;
        P->m = a.m;
        P->state_offset = 0;
        P->read_offset = 0;
        P->vinfo = vinfo;
        P->dist = dist;
        P->share = share;
        P->col = col;
        P->w = w;
        P->h = a.h;
        P->cu = a.cu;
        P->cv = a.cv;
        P->cw = a.cw;
        P->betas = a.betas;
        P->thresholds = thr;
        P->varorder = a.varorder;
        P->proposal = a.proposal;
        P->regular_degree = 0;  // general lists
        P->regular_magic = 0;
        P->resolve = 0;  // no back-neighbour records: passes end at the first dependent
        P->dense = 0;
        P->back = nullptr;
        P->bw = nullptr;
        P->dense_w = nullptr;
        P->dense_bits = nullptr;
        P->band_b = 0;
        P->band_w = 0;
    }
}

// Copies each read's near-tie count out of the fixed array (when the caller
// gave a device array for them) and sums them into the total at kOffTies.
__global__ void __launch_bounds__(1024) noalloc_ties_kernel(unsigned char *base, int num_reads,
                                                            uint32_t *out) {
    const ReadStats *stats = reinterpret_cast<const ReadStats *>(base + kOffStats);
    unsigned long long *total = reinterpret_cast<unsigned long long *>(base + kOffTies);
    __shared__ unsigned long long s_sum;
    if (threadIdx.x == 0) s_sum = 0ull;
    __syncthreads();
    unsigned long long mine = 0ull;
    for (int r = threadIdx.x; r < num_reads; r += blockDim.x) {
        const unsigned t = stats[r].near_ties;
        if (out) out[r] = t;
        mine += t;
    }
    atomicAdd(&s_sum, mine);
    __syncthreads();
    if (threadIdx.x == 0) *total = s_sum;
}

// Per-device set-up: the array's device address, the RNG jump table and the
// device properties the launch shape needs.
struct DeviceSetup {
    std::once_flag once;
    cudaError_t status = cudaSuccess;
    unsigned char *base = nullptr;
    int major = 0;
    int sms = 0;
    size_t smem_optin = 0;
};
constexpr int kMaxDevices = 64;
DeviceSetup g_setup[kMaxDevices];

uint32_t g_jump_table[kJumpTable][4];  // host copy, built once (static storage)
std::once_flag g_jump_once;

int fail(char *err, size_t errlen, int code, const std::string &msg) {
    if (err && errlen) std::snprintf(err, errlen, "%s", msg.c_str());
    return code;
}

}  // namespace
}  // namespace b200sa

using namespace b200sa;

extern "C" int b200sa_sample_noalloc(
    int32_t num_vars, const double *d_h, int64_t num_couplers, const int32_t *d_coupler_starts,
    const int32_t *d_coupler_ends, const double *d_coupler_weights, int32_t num_reads,
    const int8_t *d_states_in, int8_t *d_states_out, double *d_energies,
    int32_t sweeps_per_beta, int32_t num_betas, const double *d_beta_schedule,
    const uint64_t *d_seeds, int32_t varorder, int32_t proposal, int32_t device,
    void *stream, uint32_t *d_read_near_ties, int64_t *near_ties, char *err, size_t errlen) {
    if (near_ties) *near_ties = 0;
    // Size limits of the fixed working memory, checked before any device work.
    if (num_vars < 0 || num_couplers < 0 || num_reads < 0 || num_betas < 0 ||
        sweeps_per_beta < 0)
        return fail(err, errlen, B200SA_EINVAL, "negative size");
    if (num_vars > kNoAllocMaxVars || num_couplers > kNoAllocMaxCouplers ||
        num_betas > kNoAllocMaxBetas || num_reads > kNoAllocMaxReads) {
        char buf[256];
        std::snprintf(buf, sizeof(buf),
                      "problem exceeds the fixed working memory of b200sa_sample_noalloc "
                      "(limits: num_vars <= %lld, num_couplers <= %lld, num_betas <= %lld, "
                      "num_reads <= %lld)",
                      (long long)kNoAllocMaxVars, (long long)kNoAllocMaxCouplers,
                      (long long)kNoAllocMaxBetas, (long long)kNoAllocMaxReads);
        return fail(err, errlen, B200SA_EINVAL, buf);
    }
    if (varorder != B200SA_SEQUENTIAL && varorder != B200SA_RANDOM)
        return fail(err, errlen, B200SA_EINVAL, "varorder must be 0 or 1");
    if (proposal != B200SA_GIBBS && proposal != B200SA_METROPOLIS)
        return fail(err, errlen, B200SA_EINVAL, "proposal must be 0 or 1");
    {
        // Every call ends by waiting for its work, which a stream capture
        // does not allow: refuse before enqueuing anything.
        cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
        const cudaError_t ce = cudaStreamIsCapturing(static_cast<cudaStream_t>(stream), &cap);
        if (ce != cudaSuccess) return fail(err, errlen, B200SA_ECUDA, cudaGetErrorString(ce));
        if (cap != cudaStreamCaptureStatusNone)
            return fail(err, errlen, B200SA_EINVAL,
                        "b200sa_sample_noalloc cannot be captured into a CUDA graph: it waits "
                        "for its own work; call it outside stream capture");
    }
    if (num_reads == 0 || num_vars == 0) {
        if (num_reads && !d_energies) return fail(err, errlen, B200SA_EINVAL, "energies is NULL");
        if (num_reads) {
            cudaStream_t st = static_cast<cudaStream_t>(stream);
            cudaError_t e = cudaMemsetAsync(d_energies, 0, sizeof(double) * (size_t)num_reads, st);
            if (e == cudaSuccess && d_read_near_ties)
                e = cudaMemsetAsync(d_read_near_ties, 0, sizeof(uint32_t) * (size_t)num_reads, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) return fail(err, errlen, B200SA_ECUDA, cudaGetErrorString(e));
        }
        return num_reads;
    }
    if (!d_h || !d_states_in || !d_states_out || !d_energies || !d_seeds ||
        (num_betas && !d_beta_schedule) ||
        (num_couplers && (!d_coupler_starts || !d_coupler_ends || !d_coupler_weights)))
        return fail(err, errlen, B200SA_EINVAL, "a required device pointer is NULL");
    if (device < 0 || device >= kMaxDevices)
        return fail(err, errlen, B200SA_ENODEV, "device index out of range");

    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    struct Restore {
        int d;
        ~Restore() {
            if (d >= 0) cudaSetDevice(d);
        }
    } restore{prev};
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return fail(err, errlen, B200SA_ENODEV, cudaGetErrorString(e));

    // Once per device, with that device current: read its properties,
    // resolve the array's device address (the host-side name is only a
    // stand-in) and load the jump table.
    std::call_once(g_jump_once, [] {
        uint32_t cols[128][4];
        rng_jump_columns(kHalf, cols);
        rng_jump_nibbles(cols, g_jump_table);
    });
    DeviceSetup &S = g_setup[device];
    std::call_once(S.once, [&S, device] {
        cudaDeviceProp prop;
        S.status = cudaGetDeviceProperties(&prop, device);
        if (S.status != cudaSuccess) return;
        S.major = prop.major;
        S.sms = prop.multiProcessorCount;
        S.smem_optin = prop.sharedMemPerBlockOptin;
        if (S.major != 10) return;
        void *ptr = nullptr;
        S.status = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (S.status == cudaSuccess) S.base = static_cast<unsigned char *>(ptr);
        if (S.status == cudaSuccess) S.status = upload_jump_table(g_jump_table, nullptr);
        if (S.status == cudaSuccess) S.status = cudaStreamSynchronize(nullptr);
    });
    if (S.status == cudaSuccess && S.major != 10)
        return fail(err, errlen, B200SA_ENODEV, "this library is built for sm_100a (B200)");
    if (S.status != cudaSuccess || !S.base)
        return fail(err, errlen, B200SA_ECUDA,
                    std::string("set-up of the fixed working memory failed: ") +
                        cudaGetErrorString(S.status));

    cudaStream_t st = static_cast<cudaStream_t>(stream);
    PackArgs pa;
    pa.base = S.base;
    pa.n = num_vars;
    pa.m = num_couplers;
    pa.h = d_h;
    pa.cu = d_coupler_starts;
    pa.cv = d_coupler_ends;
    pa.cw = d_coupler_weights;
    pa.num_betas = num_betas;
    pa.betas = d_beta_schedule;
    pa.num_reads = num_reads;
    pa.sweeps_per_beta = sweeps_per_beta;
    pa.varorder = varorder;
    pa.proposal = proposal;
    noalloc_pack_kernel<<<1, 1024, 0, st>>>(pa);
    e = cudaGetLastError();
    int flag = 0;
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(&flag, S.base + kOffErr, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail(err, errlen, B200SA_ECUDA, cudaGetErrorString(e));
    if (flag)
        return fail(err, errlen, B200SA_EINVAL, "coupler indexes contain an invalid variable");

    // Launch shape: every read's state on chip (n <= 4096); most resident warps.
    const int variant = kernel_variant(
        (proposal == B200SA_GIBBS ? kKindGibbs : 0) | (varorder == B200SA_RANDOM ? kKindRandom : 0),
        kStageShared);
    const int tb = touch_bytes_for(varorder == B200SA_RANDOM, num_vars);
    const int region = region_bytes_for(num_vars) + tb;
    int best_w = 1, best = 0;
    for (int wpc = 1; wpc <= kMaxThreadsPerCta / 32; ++wpc) {
        if ((size_t)wpc * (size_t)region > S.smem_optin) break;
        int ctas = 0;
        e = kernel_occupancy(variant, wpc, region, &ctas);
        if (e != cudaSuccess) return fail(err, errlen, B200SA_ECUDA, cudaGetErrorString(e));
        if (ctas * wpc > best) {
            best = ctas * wpc;
            best_w = wpc;
        }
    }
    if (best == 0) return fail(err, errlen, B200SA_ECUDA, "kernel does not fit on an SM");
    const int wpc = (int)std::min<int64_t>(best_w, (num_reads + S.sms - 1) / S.sms);
    int ctas = 0;
    e = kernel_occupancy(variant, wpc, region, &ctas);
    if (e != cudaSuccess) return fail(err, errlen, B200SA_ECUDA, cudaGetErrorString(e));
    const int grid = (int)std::max<int64_t>(
        1, std::min<int64_t>((int64_t)S.sms * ctas, (num_reads + wpc - 1) / wpc));

    LaunchArgs a{};
    a.problems = reinterpret_cast<const ProblemDev *>(S.base + kOffProb);
    a.items = reinterpret_cast<const int64_t *>(S.base + kOffItems);
    a.num_items = num_reads;
    a.queue_head = reinterpret_cast<unsigned long long *>(S.base + kOffQueue);
    a.states_in = d_states_in;
    a.states_out = d_states_out;
    a.energies = d_energies;
    a.seeds = d_seeds;
    a.stats = reinterpret_cast<ReadStats *>(S.base + kOffStats);
    a.smem_cap_n = num_vars;
    a.touch_bytes = tb;
    e = launch_sa(variant, a, grid, wpc, region, st);
    if (e == cudaSuccess) {
        noalloc_ties_kernel<<<1, 1024, 0, st>>>(S.base, num_reads, d_read_near_ties);
        e = cudaGetLastError();
    }
    unsigned long long ties = 0ull;
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(&ties, S.base + kOffTies, sizeof(ties), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail(err, errlen, B200SA_ECUDA, cudaGetErrorString(e));
    if (near_ties) *near_ties = (int64_t)ties;
    return num_reads;
}
