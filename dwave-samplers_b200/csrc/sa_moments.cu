// Sample moments for the log-partition gradient (no reference counterpart).
//
// For p(s) proportional to exp(-beta * E(s)) with the reference's energy
// E(s) = sum_i h_i s_i + sum_c J_c s_u(c) s_v(c) (cpu_sa.cpp:210-227),
//   d log Z / d h_i = -beta <s_i>,   d log Z / d J_c = -beta <s_u(c) s_v(c)>.
// This file reduces stored samples to the integer sums sum_r s_i and
// sum_r s_u s_v per coupler (COO order).  Integer sums are exact, so the
// result does not depend on the reduction order; the caller scales them.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "b200sa.h"

namespace {

struct MomentsTile {
    int problem;
    int read0;
    int reads;
    int coupler0;   // couplers [coupler0, coupler0 + couplers) of this tile
    int couplers;
};

constexpr int kTileReads = 64;
constexpr int kTileCouplers = 8192;
constexpr int kThreads = 256;

// One block per tile: the tile's reads are streamed row by row through
// shared memory; every thread keeps running sums for its couplers in
// registers (kTileCouplers / kThreads = 32 each) and adds them to the
// problem's totals with one 64-bit atomic each.  Spin sums are added by the
// tile with coupler0 == 0.
__global__ void __launch_bounds__(kThreads)
    moments_kernel(const b200sa_moments_problem *probs, const MomentsTile *tiles) {
    extern __shared__ int8_t row[];
    const MomentsTile t = tiles[blockIdx.x];
    const b200sa_moments_problem P = probs[t.problem];
    const int n = P.num_vars;
    constexpr int kPer = kTileCouplers / kThreads;
    int acc[kPer];
#pragma unroll
    for (int j = 0; j < kPer; ++j) acc[j] = 0;
    int cu[kPer], cv[kPer];
#pragma unroll
    for (int j = 0; j < kPer; ++j) {
        const int c = t.coupler0 + j * kThreads + (int)threadIdx.x;
        const bool ok = j * kThreads + (int)threadIdx.x < t.couplers;
        cu[j] = ok ? P.coupler_starts[c] : 0;
        cv[j] = ok ? P.coupler_ends[c] : 0;
    }
    const bool spins = t.coupler0 == 0;
    int sacc[16];  // spin sums for variables threadIdx.x + k*kThreads, k < 16
#pragma unroll
    for (int k = 0; k < 16; ++k) sacc[k] = 0;
    for (int r = t.read0; r < t.read0 + t.reads; ++r) {
        const int8_t *src = P.states + (int64_t)r * n;
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += kThreads) row[i] = src[i];
        __syncthreads();
#pragma unroll
        for (int j = 0; j < kPer; ++j) acc[j] += (int)row[cu[j]] * (int)row[cv[j]];
        if (spins) {
#pragma unroll
            for (int k = 0; k < 16; ++k) {
                const int i = (int)threadIdx.x + k * kThreads;
                if (i < n) sacc[k] += row[i];
            }
        }
    }
#pragma unroll
    for (int j = 0; j < kPer; ++j) {
        const int c = t.coupler0 + j * kThreads + (int)threadIdx.x;
        if (j * kThreads + (int)threadIdx.x < t.couplers)
            atomicAdd(reinterpret_cast<unsigned long long *>(&P.sum_ss[c]),
                      (unsigned long long)(long long)acc[j]);
    }
    if (spins) {
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            const int i = (int)threadIdx.x + k * kThreads;
            if (i < n)
                atomicAdd(reinterpret_cast<unsigned long long *>(&P.sum_s[i]),
                          (unsigned long long)(long long)sacc[k]);
        }
    }
}

int fail(char *err, size_t errlen, int code, const std::string &msg) {
    if (err && errlen) std::snprintf(err, errlen, "%s", msg.c_str());
    return code;
}

}  // namespace

extern "C" int b200sa_edge_moments(const b200sa_moments_problem *problems, int32_t num_problems,
                                   int32_t device, void *stream, char *err, size_t errlen) {
    if (num_problems < 0 || (num_problems > 0 && !problems))
        return fail(err, errlen, B200SA_EINVAL, "bad problem list");
    int maxn = 0;
    std::vector<MomentsTile> tiles;
    for (int p = 0; p < num_problems; ++p) {
        const b200sa_moments_problem &q = problems[p];
        if (q.num_vars < 0 || q.num_couplers < 0 || q.num_reads < 0)
            return fail(err, errlen, B200SA_EINVAL, "negative size");
        if (q.num_vars > 16 * kThreads)
            return fail(err, errlen, B200SA_EINVAL, "num_vars above 4096");
        if (q.num_couplers > INT32_MAX)
            return fail(err, errlen, B200SA_EINVAL, "too many couplers");
        maxn = q.num_vars > maxn ? q.num_vars : maxn;
        for (int r = 0; r < q.num_reads; r += kTileReads)
            for (int64_t c = 0; c < (q.num_couplers > 0 ? q.num_couplers : 1); c += kTileCouplers)
                tiles.push_back({p, r, q.num_reads - r < kTileReads ? q.num_reads - r : kTileReads,
                                 (int)c,
                                 (int)(q.num_couplers - c < kTileCouplers ? q.num_couplers - c
                                                                          : kTileCouplers)});
    }
    if (tiles.empty()) return 0;
    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return fail(err, errlen, B200SA_ENODEV, cudaGetErrorString(e));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    b200sa_moments_problem *dprobs = nullptr;
    MomentsTile *dtiles = nullptr;
    e = cudaMallocAsync(reinterpret_cast<void **>(&dprobs),
                        sizeof(b200sa_moments_problem) * (size_t)num_problems, st);
    if (e == cudaSuccess)
        e = cudaMallocAsync(reinterpret_cast<void **>(&dtiles), sizeof(MomentsTile) * tiles.size(),
                            st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(dprobs, problems, sizeof(b200sa_moments_problem) * (size_t)num_problems,
                            cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(dtiles, tiles.data(), sizeof(MomentsTile) * tiles.size(),
                            cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        moments_kernel<<<(unsigned)tiles.size(), kThreads, (size_t)(maxn > 0 ? maxn : 1), st>>>(
            dprobs, dtiles);
        e = cudaGetLastError();
    }
    // The host arrays above must stay valid until the copies have been read.
    cudaError_t e2 = cudaStreamSynchronize(st);
    if (dprobs) cudaFreeAsync(dprobs, st);
    if (dtiles) cudaFreeAsync(dtiles, st);
    if (prev >= 0) cudaSetDevice(prev);
    if (e == cudaSuccess) e = e2;
    if (e != cudaSuccess) return fail(err, errlen, B200SA_ECUDA, cudaGetErrorString(e));
    return (int)tiles.size();
}

// ---- Counter-based initial states --------------------------------------------
// Uniform +-1 spins as a hash of (init_seed, model, read, variable): the
// splitmix64 finalizer applied to a key of (init_seed, model) and then to
// key ^ (read * 0x100000001B3 + variable); the spin is +1 when the top bit of
// the result is set.  Any range of reads regenerates identically, which is
// what lets sampled states be recomputed from seeds instead of stored.
namespace {

__device__ __forceinline__ uint64_t mix64(uint64_t x) {
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

// Each thread writes 16 consecutive spins of the flattened (reads x n) block.
__global__ void random_states_kernel(uint64_t key, int64_t read0, int64_t total, int32_t n,
                                     int8_t *out) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x * 16;
    for (int64_t base = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) * 16; base < total;
         base += stride) {
        int64_t r = base / n;
        int32_t i = (int32_t)(base - r * n);
        const int64_t end = base + 16 < total ? base + 16 : total;
        for (int64_t k = base; k < end; ++k) {
            const uint64_t x = mix64(key ^ ((uint64_t)(read0 + r) * 0x100000001B3ull + (uint64_t)i));
            out[k] = (x >> 63) ? 1 : -1;
            if (++i == n) {
                i = 0;
                ++r;
            }
        }
    }
}

}  // namespace

extern "C" int b200sa_random_states(uint64_t init_seed, uint64_t model_index, int64_t read0,
                                    int64_t num_reads, int32_t num_vars, int8_t *d_states,
                                    int32_t device, void *stream, char *err, size_t errlen) {
    if (num_reads < 0 || num_vars < 0 || read0 < 0)
        return fail(err, errlen, B200SA_EINVAL, "negative size");
    const int64_t total = num_reads * (int64_t)num_vars;
    if (total == 0) return 0;
    if (!d_states) return fail(err, errlen, B200SA_EINVAL, "null state buffer");
    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return fail(err, errlen, B200SA_ENODEV, cudaGetErrorString(e));
    const uint64_t key = [&] {
        uint64_t x = init_seed * 0x9E3779B97F4A7C15ull + model_index * 0xD1B54A32D192ED03ull;
        x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
        x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
        return x ^ (x >> 31);
    }();
    constexpr int kBlock = 256;
    const int64_t threads = (total + 15) / 16;
    int64_t blocks = (threads + kBlock - 1) / kBlock;
    if (blocks > 148 * 16) blocks = 148 * 16;
    random_states_kernel<<<(unsigned)blocks, kBlock, 0, static_cast<cudaStream_t>(stream)>>>(
        key, read0, total, num_vars, d_states);
    e = cudaGetLastError();
    if (prev >= 0) cudaSetDevice(prev);
    if (e != cudaSuccess) return fail(err, errlen, B200SA_ECUDA, cudaGetErrorString(e));
    return 0;
}
