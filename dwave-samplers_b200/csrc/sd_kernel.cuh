// Steepest descent kernel (included by sa_launch.cu, next to the annealing
// kernels whose helpers it shares).
// The drop-in for the reference's
// steepest_gradient_descent (dwave/samplers/greedy/src/descent.cpp:315-405),
// the step usually run after annealing to take every sample to a local
// minimum.  One warp per sample.
//
// Arithmetic follows descent.cpp operation for operation:
//   flip energy (descent.cpp:41-60) = -2*s * (h + sum s_nb*J, adjacency order),
//     the same expression as the annealer's delta energy (load_state);
//   selection (descent.cpp:149-156, 234-238): the least flip energy, ties to
//     the lower index, and only a negative one is taken;
//   linear-search solver (:161-182): s *= -1, fe[v] *= -1, then every list
//     entry fe[nb] -= ((4*s_new) * J) * s_nb in list order;
//   ordered-set solver (:255-285, large_sparse_opt): every list entry
//     fe[nb] += ((4*s_old) * J) * s_nb in list order, then s *= -1 and fe[v]
//     set to minus its value before the list loop;
//   state energy (:75-93) as state_energy.
// Descent stops when no flip energy is negative, or after max_steps steps:
// with a self-loop of positive weight (or spins other than +-1) a variable
// can flip back and forth for ever (the reference never returns then); here
// the sample stops at max_steps and the call reports B200SA_ETIMEOUT.
#pragma once
#include <climits>

#include "sa_kernel.cuh"

namespace b200sa {
// From this many variables on, lanes keep their minimum flip energy from step
// to step instead of rescanning (measured: 1.5x faster kernel at n = 8192;
// at n = 2048 the rescan is 1.25x faster).
constexpr int kSdCacheMinN = 4096;

// The least (energy, index) of the warp: each lane holds its own best.
__device__ __forceinline__ void warp_argmin(double &e, int &v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double oe = __shfl_xor_sync(kFull, e, o);
        const int ov = __shfl_xor_sync(kFull, v, o);
        if (oe < e || (oe == e && ov < v)) {
            e = oe;
            v = ov;
        }
    }
}

template <bool SPARSE, bool SMEM>
__global__ void __launch_bounds__(kMaxThreadsPerCta, 1)
    sd_warp_kernel(SdArgs A, int warps_per_cta, int region_bytes) {
    extern __shared__ __align__(16) uint8_t smem[];
    const unsigned lane = threadIdx.x & 31u;
    const int wid = (int)(threadIdx.x >> 5);
    uint8_t *region = smem + (size_t)wid * (size_t)region_bytes;
    double *scratch = reinterpret_cast<double *>(region);
    const int64_t gw = (int64_t)blockIdx.x * warps_per_cta + wid;
    double *fe;
    int8_t *sp;
    if (SMEM) {
        fe = reinterpret_cast<double *>(region + kSdScratchBytes);
        sp = reinterpret_cast<int8_t *>(region + kSdScratchBytes +
                                        (size_t)A.smem_cap_n * sizeof(double));
    } else {
        fe = A.scratch_fe + gw * A.scratch_stride;
        sp = A.scratch_s + gw * A.scratch_stride;
    }
    const ProblemDev *PD = A.problem;
    const Prob P = load_prob(PD);
    const int n = P.n;
    for (;;) {
        unsigned long long x = 0;
        if (lane == 0) x = atomicAdd(A.queue_head, 1ull);
        const int64_t it = (int64_t)__shfl_sync(kFull, x, 0);
        if (it >= A.num_items) break;
        const int r = (int)(A.items[it] & 0xffffffffll);
        const int64_t so = PD->state_offset + (int64_t)r * n;
        load_state(PD, A.states_in + so, fe, sp, lane);  // descent.cpp:41-60, 128-133
        // descent.cpp:149-156 / 234-238: the least flip energy below `init`,
        // ties to the lowest index.  Lane l finds that minimum (lbe, lbv) over
        // its own variables v = l (mod 32) by a scan.  For n >= kSdCacheMinN
        // the lanes keep it from step to step instead: a step changes only
        // the flipped variable and its neighbours, whose owners refresh their
        // minimum (below that size the scan of n / 32 entries is cheaper).
        const double init = SPARSE ? __longlong_as_double(0x7ff0000000000000ll) : 0.0;
        const bool cache = n >= kSdCacheMinN;
        double lbe = init;
        int lbv = INT_MAX;
        uint32_t steps = 0;
        bool capped = false;
        for (;;) {
            if (!cache || steps == 0) {
                lbe = init;
                lbv = INT_MAX;
                for (int v = lane; v < n; v += 32) {
                    const double e = fe[v];
                    if (e < lbe) {
                        lbe = e;
                        lbv = v;
                    }
                }
            }
            double be = lbe;
            int bv = lbv;
            warp_argmin(be, bv);
            if (bv == INT_MAX || !(be < 0.0)) break;  // :159-161 / :244
            if (steps >= A.max_steps) {
                capped = true;
                break;
            }
            const int s_old = (int)sp[bv];
            const int s_new = (int)(int8_t)(s_old * -1);
            __syncwarp();
            if (!SPARSE && lane == 0) {  // :168, :172
                sp[bv] = (int8_t)s_new;
                fe[bv] = __dmul_rn(fe[bv], -1.0);
            }
            __syncwarp();
            // List entries 32 at a time; equal targets within a round are
            // applied by their first lane in entry order.
            const uint2 vi = __ldg(&P.vinfo[bv]);
            const int start = (int)vi.x, deg = (int)(vi.y & kDegMask);
            const bool dup = (__ldg(&P.share[bv]) & 1u) != 0u;
            const double mult = (double)(4 * (SPARSE ? s_old : s_new));
            for (int base = 0; base < deg; base += 32) {
                const int k = base + (int)lane;
                const bool a = k < deg;
                int nb = -1 - (int)lane;
                double xk = 0.0;
                if (a) {
                    nb = __ldg(&P.col[start + k]);
                    xk = __dmul_rn(__dmul_rn(mult, __ldg(&P.w[start + k])), (double)(int)sp[nb]);
                }
                const unsigned grp = dup ? __match_any_sync(kFull, nb) : (1u << lane);
                const bool alone = grp == (1u << lane);
                if (a && alone) fe[nb] = SPARSE ? __dadd_rn(fe[nb], xk) : __dsub_rn(fe[nb], xk);
                if (dup && __any_sync(kFull, a && !alone)) {  // warp-uniform
                    scratch[lane] = xk;
                    __syncwarp();
                    if (a && !alone && lane == (unsigned)(__ffs(grp) - 1)) {
                        double acc = fe[nb];
                        unsigned g = grp;
                        while (g) {
                            const int j = __ffs(g) - 1;
                            g &= g - 1;
                            acc = SPARSE ? __dadd_rn(acc, scratch[j]) : __dsub_rn(acc, scratch[j]);
                        }
                        fe[nb] = acc;
                    }
                }
                __syncwarp();
            }
            if (SPARSE && lane == 0) {  // :280, :283-285
                sp[bv] = (int8_t)s_new;
                fe[bv] = __dmul_rn(be, -1.0);
            }
            __syncwarp();
            if (!cache) {
                ++steps;
                continue;
            }
            // The owner of every changed entry updates its minimum: a new
            // entry below it (or equal with a lower index) replaces it; its own
            // minimum entry rising above it leaves the lane to be rescanned.
            bool rescan = false;
            auto consider = [&](int x) {
                const double e = fe[x];
                if (x == lbv) {
                    if (e <= lbe)
                        lbe = e;
                    else
                        rescan = true;
                } else if (e < init && (e < lbe || (e == lbe && x < lbv))) {
                    lbe = e;
                    lbv = x;
                }
            };
            if ((bv & 31) == (int)lane) consider(bv);
            for (int base = 0; base < deg; base += 32) {
                const int k = base + (int)lane;
                const int x = k < deg ? __ldg(&P.col[start + k]) : 0;
                const int cnt = min(32, deg - base);
                for (int t = 0; t < cnt; ++t) {
                    const int xt = __shfl_sync(kFull, x, t);
                    if ((xt & 31) == (int)lane) consider(xt);
                }
            }
            // Lanes to rescan: the whole warp scans each one's variables.
            unsigned todo = __ballot_sync(kFull, rescan);
            while (todo) {
                const int L = __ffs(todo) - 1;
                todo &= todo - 1;
                double e2 = init;
                int v2 = INT_MAX;
                for (int v = L + 32 * (int)lane; v < n; v += 32 * 32) {
                    const double e = fe[v];
                    if (e < e2) {
                        e2 = e;
                        v2 = v;
                    }
                }
                warp_argmin(e2, v2);
                if ((int)lane == L) {
                    lbe = e2;
                    lbv = v2;
                }
            }
            ++steps;
        }
        __syncwarp();
        const double e = state_energy(PD, sp, lane);  // descent.cpp:75-93
        for (int v = lane; v < n; v += 32) A.states_out[so + v] = sp[v];
        if (lane == 0) {
            A.energies[PD->read_offset + r] = e;
            A.steps[PD->read_offset + r] = steps;
            if (capped) atomicAdd(A.capped, 1ull);
        }
        __syncwarp();
    }
}

}  // namespace b200sa

