// Simulated-annealing sweep for sm_100a: one warp per read.
//
// Arithmetic follows dwave-samplers 1.8.0 dwave/samplers/sa/src/cpu_sa.cpp
// operation for operation (explicit __dadd_rn/__dmul_rn, so no contraction
// can change a rounding):
//   local field / initial delta energy   cpu_sa.cpp:54-74, 113-116
//   skip threshold 44.36142/beta          cpu_sa.cpp:131, 140 (host-divided)
//   Metropolis / Gibbs acceptance         cpu_sa.cpp:144-166
//   neighbour delta-energy update         cpu_sa.cpp:172-190
//   state energy                          cpu_sa.cpp:210-227
//   xorshift128+                          cpu_sa.cpp:27-34, seeding :283-284
//
// Sequential order runs in speculative passes over a window of up to 32
// consecutive variables (one per lane).  Every lane evaluates its decision
// against the delta energies as they stand at the start of the pass; the RNG
// draw each lane would consume is placed by a prefix count of the lanes
// before it that need a draw.  A flip of variable v invalidates only lanes at
// or beyond v + dist(v), dist being the distance to v's nearest later
// neighbour, so the pass commits the prefix of lanes before the smallest such
// bound.  The committed prefix is exactly what the reference computes
// one variable at a time: its delta energies were untouched by earlier flips
// in the window and its draws land on the same stream positions.  Committed
// flips are pairwise non-adjacent; their neighbour updates are applied flip
// by flip in variable order, so additions into a shared neighbour keep the
// reference's order.
#pragma once
#include <cstdint>

#include "sa_types.h"

namespace b200sa {

__constant__ uint4 c_jump[128];  // xorshift128+ advanced by kHalf steps

constexpr unsigned kFull = 0xffffffffu;
constexpr double kTwo64 = 18446744073709551616.0;  // (double)RANDMAX
// Width of the band around an exp() decision inside which CUDA's exp and
// the host libm's exp (each within ~1 ulp of the true value) could disagree.
constexpr double kTieRel = 3.552713678800501e-15;  // 2^-48

struct RingState {
    uint64_t t0, t1;  // this lane's segment-start state for the next refill
    uint64_t q;       // outputs consumed so far (stream position, warp-uniform)
    uint64_t base;    // ring holds positions [base, base + kRing)
};

struct Counters {
    unsigned long long flips;
    unsigned long long passes;
    unsigned int near;
};

__device__ __forceinline__ void xs_advance(uint64_t &s0, uint64_t &s1) {
    uint64_t a = s0;
    const uint64_t b = s1;
    s0 = b;
    a ^= a << 23;
    s1 = a ^ b ^ (a >> 17) ^ (b >> 26);
}

__device__ __forceinline__ uint64_t xs_next(uint64_t &s0, uint64_t &s1) {
    const uint64_t b = s1;
    xs_advance(s0, s1);
    return s1 + b;
}

// State <- M * state over GF(2), M = (xorshift128+ transition)^kHalf given by
// its columns in constant memory (every lane reads the same column: broadcast).
// The column loop is only partly unrolled so the 128 column loads stay inside
// it instead of being hoisted into registers by the callers' loops.
__device__ __forceinline__ void xs_jump(uint64_t &s0, uint64_t &s1) {
    uint32_t a0 = 0, a1 = 0, a2 = 0, a3 = 0;
#pragma unroll 1
    for (int k = 0; k < 4; ++k) {
        const uint32_t w = (uint32_t)((k < 2 ? s0 : s1) >> ((k & 1) * 32));
#pragma unroll 8
        for (int b = 0; b < 32; ++b) {
            const uint32_t mk = 0u - ((w >> b) & 1u);
            const uint4 c = c_jump[k * 32 + b];
            a0 ^= c.x & mk;
            a1 ^= c.y & mk;
            a2 ^= c.z & mk;
            a3 ^= c.w & mk;
        }
    }
    s0 = (uint64_t)a0 | ((uint64_t)a1 << 32);
    s1 = (uint64_t)a2 | ((uint64_t)a3 << 32);
}

// Lane l writes stream positions pos + l*kPerLane + t, t < kPerLane, starting
// from the state that precedes position pos + l*kPerLane.
__device__ __forceinline__ void ring_fill(uint64_t *ring, uint64_t pos,
                                          uint64_t s0, uint64_t s1,
                                          unsigned lane) {
    const uint64_t start = pos + (uint64_t)lane * kPerLane;
#pragma unroll
    for (int t = 0; t < kPerLane; ++t)
        ring[(start + t) & (kRing - 1)] = xs_next(s0, s1);
}

__device__ __forceinline__ void ring_init(uint64_t *ring, RingState &rs,
                                          uint64_t seed, unsigned lane) {
    uint64_t s0 = seed ? seed : ~0ull, s1 = 0;  // cpu_sa.cpp:283-284
    for (unsigned k = 0; k < lane * kPerLane; ++k) xs_advance(s0, s1);
    __syncwarp();
    ring_fill(ring, 0, s0, s1, lane);
    xs_jump(s0, s1);
    ring_fill(ring, kHalf, s0, s1, lane);
    xs_jump(s0, s1);
    rs.t0 = s0;
    rs.t1 = s1;
    rs.q = 0;
    rs.base = 0;
    __syncwarp();
}

// Keeps positions [q, q + kHalf) available: once the lower half is consumed
// it is overwritten with the positions kRing further on.
__device__ __forceinline__ void ring_refill(uint64_t *ring, RingState &rs,
                                            unsigned lane) {
    if (rs.q - rs.base >= (uint64_t)kHalf) {
        __syncwarp();
        ring_fill(ring, rs.base + kRing, rs.t0, rs.t1, lane);
        xs_jump(rs.t0, rs.t1);
        rs.base += kHalf;
        __syncwarp();
    }
}

// cpu_sa.cpp:54-74 for every variable, then the working copy of the spins.
__device__ __forceinline__ void load_state(const ProblemDev &P,
                                           const int8_t *src, double *de,
                                           int8_t *sp, unsigned lane) {
    const int n = P.n;
    for (int v = lane; v < n; v += 32) sp[v] = src[v];
    __syncwarp();
    for (int v = lane; v < n; v += 32) {
        double f = __ldg(&P.h[v]);
        const int e1 = __ldg(&P.row[v + 1]);
        for (int e = __ldg(&P.row[v]); e < e1; ++e)
            f = __dadd_rn(f, __dmul_rn((double)(int)sp[__ldg(&P.col[e])],
                                       __ldg(&P.w[e])));
        de[v] = __dmul_rn((double)(-2 * (int)sp[v]), f);
    }
    __syncwarp();
}

// cpu_sa.cpp:168-191 for variable v.  Distinct neighbour slots are updated
// lane-parallel; a list with repeated targets runs on one lane in order.
__device__ __forceinline__ void apply_flip(const ProblemDev &P, double *de,
                                           int8_t *sp, int v, unsigned lane) {
    const int s_old = sp[v];
    const double mult = (double)(int)(int8_t)(4 * s_old);
    const int e0 = __ldg(&P.row[v]), e1 = __ldg(&P.row[v + 1]);
    if (!(__ldg(&P.vinfo[v]) & kDupFlag)) {
        for (int e = e0 + (int)lane; e < e1; e += 32) {
            const int nb = __ldg(&P.col[e]);
            const double upd = __dmul_rn(__dmul_rn(mult, __ldg(&P.w[e])),
                                         (double)(int)sp[nb]);
            de[nb] = __dadd_rn(de[nb], upd);
        }
    } else if (lane == 0) {
        for (int e = e0; e < e1; ++e) {
            const int nb = __ldg(&P.col[e]);
            const double upd = __dmul_rn(__dmul_rn(mult, __ldg(&P.w[e])),
                                         (double)(int)sp[nb]);
            de[nb] = __dadd_rn(de[nb], upd);
        }
    }
    __syncwarp();
    if (lane == 0) {
        sp[v] = (int8_t)(-s_old);
        de[v] = __dmul_rn(de[v], -1.0);
    }
    __syncwarp();
}

template <bool GIBBS>
__device__ __forceinline__ void sweep_sequential(const ProblemDev &P,
                                                 double *de, int8_t *sp,
                                                 uint64_t *ring, RingState &rs,
                                                 unsigned lane, Counters &cnt) {
    const int n = P.n;
    const unsigned lt_mask = (1u << lane) - 1u;
    for (int b = 0; b < P.num_betas; ++b) {
        const double beta = __ldg(&P.betas[b]);
        const double thr = __ldg(&P.thresholds[b]);
        for (int sw = 0; sw < P.sweeps_per_beta; ++sw) {
            int p = 0;
            while (p < n) {
                ring_refill(ring, rs, lane);
                const int L = min(32, n - p);
                const int v = p + (int)lane;
                const bool act = (int)lane < L;
                const double d = act ? de[v] : 0.0;
                const int dist = act ? (int)(__ldg(&P.vinfo[v]) & kDistMask) : 32;
                const bool consider = act && !(d >= thr);  // cpu_sa.cpp:140
                const bool need = GIBBS ? consider : (consider && !(d <= 0.0));
                const unsigned need_mask = __ballot_sync(kFull, need);
                bool acc = GIBBS ? false : consider;  // Metropolis: d <= 0 accepts
                bool near = false;
                if (need) {
                    const uint64_t r =
                        ring[(rs.q + (uint64_t)__popc(need_mask & lt_mask)) &
                             (kRing - 1)];
                    const double rd = __ull2double_rn(r);
                    if (GIBBS) {  // cpu_sa.cpp:162-163
                        const double e = exp(__dmul_rn(d, beta));
                        const double y = __dmul_rn(rd, __dadd_rn(1.0, e));
                        acc = kTwo64 > y;
                        near = fabs(y - kTwo64) <= kTwo64 * kTieRel;
                    } else {  // cpu_sa.cpp:152-154
                        const double e = exp(__dmul_rn(-d, beta));
                        const double x = __dmul_rn(e, kTwo64);
                        acc = x > rd;
                        near = fabs(x - rd) <= x * kTieRel;
                    }
                }
                const unsigned flip_mask = __ballot_sync(kFull, acc);
                const int bound = acc ? (int)lane + dist : 32;
                const int c = min(__reduce_min_sync(kFull, bound), L);
                const unsigned commit = c >= 32 ? kFull : ((1u << c) - 1u);
                rs.q += (uint64_t)__popc(need_mask & commit);
                cnt.near += __popc(__ballot_sync(kFull, near) & commit);
                unsigned fm = flip_mask & commit;
                cnt.flips += __popc(fm);
                cnt.passes += 1;
                while (fm) {
                    const int k = __ffs(fm) - 1;
                    fm &= fm - 1;
                    apply_flip(P, de, sp, p + k, lane);
                }
                p += c;
            }
        }
    }
}

// cpu_sa.cpp:134-136: each attempt draws its variable as rand % n.  One
// attempt per step, warp-uniform; lanes share the neighbour update.
template <bool GIBBS>
__device__ __forceinline__ void sweep_random(const ProblemDev &P, double *de,
                                             int8_t *sp, uint64_t *ring,
                                             RingState &rs, unsigned lane,
                                             Counters &cnt) {
    const int n = P.n;
    for (int b = 0; b < P.num_betas; ++b) {
        const double beta = __ldg(&P.betas[b]);
        const double thr = __ldg(&P.thresholds[b]);
        for (int sw = 0; sw < P.sweeps_per_beta; ++sw) {
            for (int i = 0; i < n; ++i) {
                ring_refill(ring, rs, lane);
                const uint64_t r1 = ring[rs.q & (kRing - 1)];
                rs.q += 1;
                const int var = (int)(r1 % (uint64_t)n);
                const double d = de[var];
                cnt.passes += 1;
                if (d >= thr) continue;
                bool acc;
                if (GIBBS) {
                    const double rd = __ull2double_rn(ring[rs.q & (kRing - 1)]);
                    rs.q += 1;
                    const double y =
                        __dmul_rn(rd, __dadd_rn(1.0, exp(__dmul_rn(d, beta))));
                    acc = kTwo64 > y;
                    cnt.near += fabs(y - kTwo64) <= kTwo64 * kTieRel;
                } else if (d <= 0.0) {
                    acc = true;
                } else {
                    const double rd = __ull2double_rn(ring[rs.q & (kRing - 1)]);
                    rs.q += 1;
                    const double x = __dmul_rn(exp(__dmul_rn(-d, beta)), kTwo64);
                    acc = x > rd;
                    cnt.near += fabs(x - rd) <= x * kTieRel;
                }
                __syncwarp();
                if (acc) {
                    cnt.flips += 1;
                    apply_flip(P, de, sp, var, lane);
                }
            }
        }
    }
}

// cpu_sa.cpp:210-227.  Terms are formed lane-parallel (products are exact
// roundings of the same operands); the running sum is strictly sequential.
__device__ __forceinline__ double state_energy(const ProblemDev &P,
                                               const int8_t *sp,
                                               unsigned lane) {
    double e = 0.0;
    for (int base = 0; base < P.n; base += 32) {
        const int v = base + (int)lane;
        const double t =
            v < P.n ? __dmul_rn((double)(int)sp[v], __ldg(&P.h[v])) : 0.0;
        const int cnt = min(32, P.n - base);
        for (int j = 0; j < cnt; ++j) e = __dadd_rn(e, __shfl_sync(kFull, t, j));
    }
    for (int64_t base = 0; base < P.m; base += 32) {
        const int64_t c = base + lane;
        double t = 0.0;
        if (c < P.m)
            t = __dmul_rn(__dmul_rn((double)(int)sp[__ldg(&P.cu[c])], __ldg(&P.cw[c])),
                          (double)(int)sp[__ldg(&P.cv[c])]);
        const int cnt = (int)min((int64_t)32, P.m - base);
        for (int j = 0; j < cnt; ++j) e = __dadd_rn(e, __shfl_sync(kFull, t, j));
    }
    return e;
}

template <bool GIBBS, bool RANDOM_ORDER>
__device__ __forceinline__ void anneal_read(const ProblemDev &P,
                                            const int8_t *src, int8_t *dst,
                                            double *energy_out, double *de,
                                            int8_t *sp, uint64_t *ring,
                                            RingState &rs, unsigned lane,
                                            Counters &cnt) {
    load_state(P, src, de, sp, lane);
    if (RANDOM_ORDER)
        sweep_random<GIBBS>(P, de, sp, ring, rs, lane, cnt);
    else
        sweep_sequential<GIBBS>(P, de, sp, ring, rs, lane, cnt);
    __syncwarp();
    const double e = state_energy(P, sp, lane);
    for (int v = lane; v < P.n; v += 32) dst[v] = sp[v];
    if (lane == 0) *energy_out = e;
    __syncwarp();
}

template <bool SMEM>
__device__ __forceinline__ void anneal_dispatch(const ProblemDev &P,
                                                const int8_t *src, int8_t *dst,
                                                double *energy_out, double *de,
                                                int8_t *sp, uint64_t *ring,
                                                RingState &rs, unsigned lane,
                                                Counters &cnt) {
    const bool gibbs = P.proposal == 0;
    if (P.varorder == 0) {
        if (gibbs)
            anneal_read<true, false>(P, src, dst, energy_out, de, sp, ring, rs, lane, cnt);
        else
            anneal_read<false, false>(P, src, dst, energy_out, de, sp, ring, rs, lane, cnt);
    } else {
        if (gibbs)
            anneal_read<true, true>(P, src, dst, energy_out, de, sp, ring, rs, lane, cnt);
        else
            anneal_read<false, true>(P, src, dst, energy_out, de, sp, ring, rs, lane, cnt);
    }
}

}  // namespace b200sa
