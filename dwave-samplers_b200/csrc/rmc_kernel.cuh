// Rotor-model annealing (the reference's SQA rotor Monte Carlo,
// dwave/samplers/sqa/src/cpu_rotormc.cpp) on the GPU.  Included by
// sa_launch.cu next to the annealing kernels.
//
// One thread per read.  The proposals MetropolisUniform and MetropolisTF
// recompute the local field on every attempt and draw a data-dependent
// number of random numbers, so a read is one sequential chain; many reads run
// side by side instead.  States and delta energies are interleaved across
// reads (element (v, r) at v * R + r), so in sequential order the 32 reads of
// a warp touch one variable in one transaction.  Each thread copies its
// sample's row of the caller's row-major states into that layout first and
// back at the end.
//
// Arithmetic follows cpu_rotormc.cpp operation for operation:
//   local field (:46-60)       h + cos(theta_nb) * J, adjacency order
//   non-ergodic delta (:130-139) field * (-2 * cos(theta))
//   burn-in (:141-143)         32 draws before the first sweep of every run
//   Metropolis / Gibbs (:167-196), uniform and transverse-field proposals
//   (:197-266), updates (:268-287), statistics (:289-293), energy (:310-326).
// cos / |sin| of the 256 angles come from the host (cpu_rotormc.cpp:377-383,
// the host libm), copied into shared memory.
#pragma once
#include "sa_kernel.cuh"

namespace b200sa {

// Metropolis-type decision exp(x) * 2^64 > (double)r, counting draws within
// the cross-libm tie band.
__device__ __forceinline__ bool rmc_metropolis(double x, uint64_t r, unsigned &near) {
    const double e = __dmul_rn(exp(x), kTwo64);
    const double rd = __ull2double_rn(r);
    near += fabs(e - rd) <= e * kTieRel;
    return e > rd;
}

template <bool RANDOM_ORDER, int PROPOSAL>
__global__ void __launch_bounds__(64) rmc_kernel(RmcArgs A) {
    __shared__ double cs[256], sn[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) {
        cs[i] = A.cos_table[i];
        sn[i] = A.sin_table[i];
    }
    __syncthreads();
    const int R = A.num_samples;
    const int n = A.n;
    const int first = A.shared_stream ? 0 : (int)(blockIdx.x * blockDim.x + threadIdx.x);
    if (first >= R) return;
    if (A.shared_stream && (blockIdx.x != 0 || threadIdx.x != 0)) return;
    const int last = A.shared_stream ? R : first + 1;
    const int points = A.interval ? 1 + (A.num_betas - 1) / A.interval : 0;
    uint64_t rng[2] = {0, 0};
    unsigned near = 0;
    for (int r = first; r < last; ++r) {
        if (!A.shared_stream || r == 0) {  // cpu_rotormc.cpp:389-390
            rng[0] = A.seeds[A.shared_stream ? 0 : r] ? A.seeds[A.shared_stream ? 0 : r] : ~0ull;
            rng[1] = 0;
        }
        const int64_t R64 = R;
        uint8_t *st = A.states + r;  // element v at st[v * R]
        double *de = A.de + r;
        uint8_t *row = A.rows + (int64_t)r * n;
        for (int v = 0; v < n; ++v) st[v * R64] = row[v];
        auto field = [&](int var) {
            const uint2 vi = __ldg(&A.vinfo[var]);
            double e = __ldg(&A.h[var]);
            for (unsigned k = vi.x; k < vi.x + vi.y; ++k)
                e = __dadd_rn(e, __dmul_rn(cs[st[(int64_t)__ldg(&A.col[k]) * R64]], __ldg(&A.w[k])));
            return e;
        };
        for (int v = 0; v < n; ++v) {
            double e = field(v);
            if (PROPOSAL <= 1) e = __dmul_rn(e, __dmul_rn(-2.0, cs[st[v * R64]]));
            de[v * R64] = e;
        }
        for (int i = 0; i < 32; ++i) xs_advance(rng[0], rng[1]);  // burn-in
        uint8_t *stats = A.stats ? A.stats + (int64_t)r * points * n : nullptr;
        for (int b = 0; b < A.num_betas; ++b) {
            const double beta = __ldg(&A.hp[b]);
            const double beta_tf = __ldg(&A.hd[b]);
            const double rat = __ddiv_rn(beta_tf, beta);
            for (int sw = 0; sw < A.sweeps_per_beta; ++sw) {
                for (int i = 0; i < n; ++i) {
                    int var = i;
                    if (RANDOM_ORDER) var = (int)(xs_next(rng[0], rng[1]) % (uint64_t)n);
                    const uint8_t cur = st[var * R64];
                    uint8_t prop;
                    double prop_e;
                    bool flip = false;
                    if (PROPOSAL == 1) {  // MetropolisNonErgodic
                        const double d = de[var * R64];
                        prop = (uint8_t)(128 + cur);
                        prop_e = -d;
                        if (d <= 0.0)
                            flip = true;
                        else
                            flip = rmc_metropolis(__dmul_rn(-d, beta), xs_next(rng[0], rng[1]), near);
                    } else if (PROPOSAL == 0) {  // GibbsNonErgodic
                        const double d = de[var * R64];
                        prop = (uint8_t)(128 + cur);
                        prop_e = -d;
                        const double y = __dmul_rn(__ull2double_rn(xs_next(rng[0], rng[1])),
                                                   __dadd_rn(1.0, exp(__dmul_rn(d, beta))));
                        near += fabs(y - kTwo64) <= kTwo64 * kTieRel;
                        flip = kTwo64 > y;
                    } else {
                        uint64_t r1 = xs_next(rng[0], rng[1]);
                        if (PROPOSAL == 2 || rat >= 1) {
                            prop = (uint8_t)(r1 % 256);
                        } else {  // MetropolisTF, cpu_rotormc.cpp:208-233
                            const int osi = (int)__dsub_rn(__dmul_rn(rat, 128.0), 0.5);
                            const double distc = __ddiv_rn((double)(osi * (osi + 1)),
                                                           (double)(2 * osi + 1));
                            const double p = __ddiv_rn(
                                __dsub_rn(__dmul_rn(__ddiv_rn(rat, 2.0), 128.0), distc),
                                __dsub_rn((double)(osi + 1), distc));
                            const uint64_t rl = r1;
                            r1 = xs_next(rng[0], rng[1]);
                            const uint8_t pac =
                                __dmul_rn(p, kTwo64) > __ull2double_rn(rl)
                                    ? (uint8_t)((uint64_t)(osi + 1) * (2 * (r1 % 2) - 1))
                                    : (uint8_t)(r1 % (uint64_t)(2 * osi + 1) - (uint64_t)osi);
                            prop = (uint8_t)(cur + pac);
                        }
                        prop_e = field(var);
                        const double dlm = __dadd_rn(
                            __dmul_rn(__dmul_rn(-beta, prop_e), __dsub_rn(cs[prop], cs[cur])),
                            __dmul_rn(__dmul_rn(beta_tf, __ldg(&A.tf[var])),
                                      __dsub_rn(sn[prop], sn[cur])));
                        if (dlm >= 0.0)
                            flip = true;
                        else
                            flip = rmc_metropolis(dlm, xs_next(rng[0], rng[1]), near);
                    }
                    if (flip) {
                        if (PROPOSAL <= 1) {  // :270-283
                            const double mult = __dmul_rn(2.0, __dsub_rn(cs[cur], cs[prop]));
                            const uint2 vi = __ldg(&A.vinfo[var]);
                            for (unsigned k = vi.x; k < vi.x + vi.y; ++k) {
                                const int64_t nb = (int64_t)__ldg(&A.col[k]) * R64;
                                de[nb] = __dadd_rn(de[nb], __dmul_rn(__dmul_rn(mult, __ldg(&A.w[k])),
                                                                     cs[st[nb]]));
                            }
                            de[var * R64] = prop_e;
                        }
                        st[var * R64] = prop;
                    }
                }
            }
            if (stats && b % A.interval == 0) {
                for (int v = 0; v < n; ++v) stats[v] = st[v * R64];
                stats += n;
            }
        }
        double e = 0.0;  // cpu_rotormc.cpp:310-326
        for (int v = 0; v < n; ++v) e = __dadd_rn(e, __dmul_rn(cs[st[v * R64]], __ldg(&A.h[v])));
        for (int64_t c = 0; c < A.m; ++c)
            e = __dadd_rn(e, __dmul_rn(__dmul_rn(cs[st[(int64_t)__ldg(&A.cu[c]) * R64]], __ldg(&A.cw[c])),
                                       cs[st[(int64_t)__ldg(&A.cv[c]) * R64]]));
        A.energies[r] = e;
        for (int v = 0; v < n; ++v) row[v] = st[v * R64];
    }
    if (near) atomicAdd(A.near, (unsigned long long)near);
}

}  // namespace b200sa
