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
// in the window and its draws land on the same stream positions.
//
// Committed flips are pairwise non-adjacent, so their neighbour updates never
// touch each other's slots or spins.  They are applied together: the
// adjacency entries of all committed flips, concatenated in variable order,
// are spread over the lanes 32 at a time.  Entries that name the same slot
// (a neighbour shared by two flips, or a self-loop / repeated coupler) are
// grouped with __match_any_sync and added by the group's first lane in entry
// order, so every slot receives its additions in the reference's order.  The
// grouping is skipped when the per-variable conflict masks (computed at pack
// time) show that no two entries of the pass can name the same slot.  Slots in
// global memory receive their additions as L2 reductions (see GlobalDe).
#pragma once
#include <cstdint>

#include "sa_types.h"

namespace b200sa {

// Nibble tables of the GF(2) matrix (xorshift128+ transition)^kHalf.
__device__ uint4 g_jump_nib[kJumpTable];

constexpr unsigned kFull = 0xffffffffu;
constexpr double kTwo64 = 18446744073709551616.0;  // (double)RANDMAX
// Width of the band around an exp() decision inside which CUDA's exp and
// the host libm's exp (each within ~1 ulp of the true value) could disagree.
constexpr double kTieRel = 3.552713678800501e-15;  // 2^-48

// Stream positions are kept modulo 2^32: only their differences (all below
// kRing) and their residues modulo kRing are used, and both survive the wrap.
struct RingState {
    uint32_t q;     // outputs consumed so far (stream position, warp-uniform)
    uint32_t base;  // ring holds positions [base, base + kRing)
};

// Per-warp words the sweep loop touches rarely, kept in the warp's shared
// region after the conflict scratch (kColdBytes): each lane's segment-start
// state for the next ring refill (once per kHalf draws) and the read's
// counters (added to by lane 0 once per sweep).  Every member is accessed
// with 8-byte (or smaller) loads and stores, so the region needs only the
// 8-byte alignment of the ring before it.
struct WarpCold {
    uint64_t seg[64];  // lane l: words 2l, 2l + 1
    unsigned long long flips;
    unsigned long long passes;
    unsigned int near;
    unsigned int pad[3];
};
static_assert(sizeof(WarpCold) == kColdBytes, "cold words");

// The ring is followed by the scratch (kScratchHotBytes), then WarpCold.
__device__ __forceinline__ WarpCold *warp_cold(uint64_t *ring) {
    return reinterpret_cast<WarpCold *>(reinterpret_cast<uint8_t *>(ring + kRing) +
                                        kScratchHotBytes);
}

// One sweep's counts (warp-uniform; at most n each), added by lane 0 to the
// read's counters when the sweep ends.
struct SweepCount {
    unsigned flips = 0, passes = 0, near = 0;
    __device__ __forceinline__ void pass(unsigned f, unsigned nt) {
        flips += f;
        passes += 1;
        near += nt;
    }
    __device__ __forceinline__ void flush(uint64_t *ring, unsigned lane) const {
        if (lane == 0) {
            WarpCold *c = warp_cold(ring);
            c->flips += flips;
            c->passes += passes;
            c->near += near;
        }
    }
};

// ---- acceptance tests ------------------------------------------------------
// The reference decides Metropolis as exp(x) * 2^64 > (double)rand with
// x = -dE*beta (cpu_sa.cpp:154) and Gibbs as 2^64 > (double)rand * (1 +
// exp(z)) with z = dE*beta (cpu_sa.cpp:163).  Both are first decided in the
// log2 domain with single-precision hardware approximations, whose total
// error is below 2^-14 in log2 units for the argument ranges that reach them
// (|x| < 44.4 and z < 44.4 since dE < 44.36142/beta): every term's error is
// bounded by a few single-precision roundings of magnitudes <= 110 plus the
// lg2/ex2 approximation error (relative 2^-22).  When the two sides differ by
// more than kBand = 2^-10 the fast answer equals the exact one; otherwise the
// exact double-precision expression is evaluated.  The band is reached by
// about 0.1% of draws.
constexpr float kLog2e = 1.4426950408889634f;
constexpr float kBand = 0.0009765625f;  // 2^-10

__device__ __forceinline__ float lg2_approx(float x) {
    float r;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

__device__ __forceinline__ float ex2_approx(float x) {
    float r;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// 1 accept, 0 reject, -1 undecided.  x = -dE*beta in (-44.4, 0].
__device__ __forceinline__ int metropolis_fast(double x, uint64_t r) {
    const float t = __fmaf_rn((float)x, kLog2e, 64.0f);  // log2(exp(x) * 2^64)
    const float y = lg2_approx(__ull2float_rn(r));      // log2(rand); -inf at 0
    if (t > y + kBand) return 1;
    if (t < y - kBand) return 0;
    return -1;
}

// 1 accept, 0 reject, -1 undecided.  z = dE*beta < 44.4 (may be -inf).
__device__ __forceinline__ int gibbs_fast(double z, uint64_t r) {
    const float zf = (float)z;
    float g;  // log2(1 + exp(z))
    if (zf > 24.0f)
        g = zf * kLog2e;  // log2(1 + exp(-z)) < 2^-33 omitted
    else if (zf < -24.0f)
        g = 0.0f;  // log2(1 + exp(z)) < 2^-33
    else
        g = lg2_approx(1.0f + ex2_approx(zf * kLog2e));
    const float s = lg2_approx(__ull2float_rn(r)) + g;  // log2(rand * (1 + exp(z)))
    if (s < 64.0f - kBand) return 1;
    if (s > 64.0f + kBand) return 0;
    return -1;
}

// The exact double-precision decisions, reached only inside the band.  Kept
// out of line so the sweep loop does not hold exp()'s registers.
// Returns accept in bit 0 and the near-tie flag in bit 1.
__device__ __noinline__ int metropolis_exact(double d, double beta, uint64_t r) {
    const double rd = __ull2double_rn(r);
    const double e = exp(__dmul_rn(-d, beta));  // cpu_sa.cpp:152-154
    const double x = __dmul_rn(e, kTwo64);
    return (x > rd ? 1 : 0) | (fabs(x - rd) <= x * kTieRel ? 2 : 0);
}

__device__ __noinline__ int gibbs_exact(double d, double beta, uint64_t r) {
    const double rd = __ull2double_rn(r);
    const double e = exp(__dmul_rn(d, beta));  // cpu_sa.cpp:162-163
    const double y = __dmul_rn(rd, __dadd_rn(1.0, e));
    return (kTwo64 > y ? 1 : 0) | (fabs(y - kTwo64) <= kTwo64 * kTieRel ? 2 : 0);
}

// A field of the problem record read again at each use, for values used once
// per sweep that are not worth a register through the sweep loop.  The load
// goes through the read-only cache (ld.global.nc, an L1 hit after the first
// sweep); the asm statement is volatile so that the compiler does not hoist
// it out of the loop.  The record does not change while a kernel runs.
__device__ __forceinline__ int reload(const int &x) {
    int r;
    asm volatile("ld.global.nc.s32 %0, [%1];" : "=r"(r) : "l"(&x));
    return r;
}
template <class T>
__device__ __forceinline__ T *reload(T *const &x) {
    unsigned long long r;
    asm volatile("ld.global.nc.u64 %0, [%1];" : "=l"(r) : "l"(&x));
    return reinterpret_cast<T *>(r);
}

// Problem fields the sweep loop keeps in registers (fields used only when a
// read starts or ends are read from the ProblemDev record there).
struct Prob {
    int n;
    const ProblemDev *pd;  // the schedule is read from here once per beta
    const uint2 *__restrict__ vinfo;
    const int32_t *__restrict__ col;
    const double *__restrict__ w;
    const uint8_t *__restrict__ dist;
    const uint32_t *__restrict__ share;
    int regular_degree;
    uint32_t regular_magic;
    const uint2 *__restrict__ back;
    const double *__restrict__ bw;
    const double *__restrict__ dense_w;
    const uint32_t *__restrict__ dense_bits;
    int dense;
};

__device__ __forceinline__ Prob load_prob(const ProblemDev *P) {
    Prob q;
    q.n = P->n;
    q.pd = P;
    q.vinfo = P->vinfo;
    q.col = P->col;
    q.w = P->w;
    q.dist = P->dist;
    q.share = P->share;
    q.regular_degree = P->regular_degree;
    q.regular_magic = P->regular_magic;
    q.back = P->back;
    q.bw = P->bw;
    q.dense_w = P->dense_w;
    q.dense_bits = P->dense_bits;
    q.dense = P->dense;
    return q;
}

// Brings the line holding *p (global memory) into L1 without waiting.
__device__ __forceinline__ void prefetch_l1(const void *p) {
    asm volatile("prefetch.global.L1 [%0];" : : "l"(p));
}

// Accessors of a read's delta energies, one per state location: get, set and
// add (de[x] = de[x] + v, rounded to nearest like the reference's `+=`,
// cpu_sa.cpp:172-185).  kAsyncAdd: an add does not wait for memory.
//
// SharedDe: the warp's shared region (kStageShared).
struct SharedDe {
    static constexpr bool kAsyncAdd = false;
    double *p;
    __device__ __forceinline__ double get(int x) const { return p[x]; }
    __device__ __forceinline__ void set(int x, double v) const { p[x] = v; }
    __device__ __forceinline__ void add(int x, double v) const { p[x] = __dadd_rn(p[x], v); }
};

// GlobalDe: the warp's global slot (kStageGlobal, kStageSpins), L2-resident.
// An add is a reduction performed at L2 (red.global.add.f64, round to
// nearest even, the same rounding as a load, __dadd_rn and a store), so the
// update phase issues its additions without waiting for the slots' values.
// Two adds to one slot from one thread land in program order, and a barrier
// of the warp orders them before any later access by its lanes.  Reads go to
// L2 (ld.global.cg), where the reductions are performed, never to a line an
// earlier read left in L1.
struct GlobalDe {
    static constexpr bool kAsyncAdd = true;
    double *p;
    __device__ __forceinline__ double get(int x) const { return __ldcg(p + x); }
    __device__ __forceinline__ void set(int x, double v) const { __stcg(p + x, v); }
    __device__ __forceinline__ void add(int x, double v) const {
        asm volatile("red.global.add.f64 [%0], %1;" : : "l"(p + x), "d"(v) : "memory");
    }
};

// BandDe: a banded problem (kStageBand).  The slots of the variables in
// [lo, lo + w) live in a shared-memory ring (`b`, w a power of two, slot
// x & (w - 1)); every other variable's slot is in the global array `g`.  The
// band slides with the window (see sweep_sequential) and fetches its slots
// with cp.async through L1, so the global part is read and written with plain
// loads and stores.  With w = 0 everything is global.
struct BandDe {
    static constexpr bool kAsyncAdd = false;
    double *g;
    double *b;
    int lo;
    unsigned w;
    __device__ __forceinline__ double &at(int x) const {
        return (unsigned)(x - lo) < w ? b[(unsigned)x & (w - 1u)] : g[x];
    }
    __device__ __forceinline__ double get(int x) const { return at(x); }
    __device__ __forceinline__ void set(int x, double v) const { at(x) = v; }
    __device__ __forceinline__ void add(int x, double v) const {
        double &s = at(x);
        s = __dadd_rn(s, v);
    }
};

template <int STAGE>
struct DeFor {
    using T = GlobalDe;
};
template <>
struct DeFor<kStageShared> {
    using T = SharedDe;
};
template <>
struct DeFor<kStageBand> {
    using T = BandDe;
};

// 8-byte asynchronous copy global -> shared (completes at cp_async_wait).
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" : : "r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;" : : : "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" : : "n"(N) : "memory");
}

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

// State <- M * state over GF(2), M = (xorshift128+ transition)^kHalf: the
// XOR of one table entry per nibble of the 128-bit state (32 lookups).
__device__ __forceinline__ void xs_jump(uint64_t &s0, uint64_t &s1) {
    uint32_t a0 = 0, a1 = 0, a2 = 0, a3 = 0;
#pragma unroll
    for (int k = 0; k < kJumpNibbles; ++k) {
        const uint64_t word = k < 16 ? s0 : s1;
        const uint32_t nib = (uint32_t)(word >> (4 * (k & 15))) & 15u;
        const uint4 c = __ldg(&g_jump_nib[k * 16 + nib]);
        a0 ^= c.x;
        a1 ^= c.y;
        a2 ^= c.z;
        a3 ^= c.w;
    }
    s0 = (uint64_t)a0 | ((uint64_t)a1 << 32);
    s1 = (uint64_t)a2 | ((uint64_t)a3 << 32);
}

// Lane l writes stream positions pos + l*kPerLane + t, t < kPerLane, starting
// from the state that precedes position pos + l*kPerLane.
__device__ __forceinline__ void ring_fill(uint64_t *ring, uint32_t pos,
                                          uint64_t s0, uint64_t s1,
                                          unsigned lane) {
    const uint32_t start = pos + lane * (uint32_t)kPerLane;
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
    uint64_t *seg = warp_cold(ring)->seg + 2 * lane;
    seg[0] = s0;
    seg[1] = s1;
    rs.q = 0;
    rs.base = 0;
    __syncwarp();
}

// Overwrites the consumed lower half with the positions kRing further on and
// advances this lane's segment-start state.  Out of line: it runs once per
// kHalf draws.
__device__ __noinline__ void ring_refill_half(uint64_t *ring, uint32_t pos, unsigned lane) {
    __syncwarp();
    uint64_t *seg = warp_cold(ring)->seg + 2 * lane;
    uint64_t s0 = seg[0], s1 = seg[1];
    ring_fill(ring, pos, s0, s1, lane);
    xs_jump(s0, s1);
    seg[0] = s0;
    seg[1] = s1;
    __syncwarp();
}

// Keeps positions [q, q + kHalf) available: once the lower half is consumed
// it is overwritten with the positions kRing further on.
__device__ __forceinline__ void ring_refill(uint64_t *ring, RingState &rs,
                                            unsigned lane) {
    if (rs.q - rs.base >= (uint32_t)kHalf) {
        ring_refill_half(ring, rs.base + kRing, lane);
        rs.base += kHalf;
    }
}

// cpu_sa.cpp:54-74 for every variable, then the working copy of the spins.
// Returns (warp-uniform) whether every spin is +1 or -1.
__device__ __forceinline__ bool load_state(const ProblemDev *PD, const int8_t *src,
                                           double *de, int8_t *sp,
                                           unsigned lane) {
    const int n = PD->n;
    const uint2 *__restrict__ vinfo = PD->vinfo;
    const int32_t *__restrict__ col = PD->col;
    const double *__restrict__ w = PD->w;
    const double *__restrict__ h = PD->h;
    bool pm1 = true;
    for (int v = lane; v < n; v += 32) {
        const int8_t x = src[v];
        sp[v] = x;
        pm1 = pm1 && (x == 1 || x == -1);
    }
    pm1 = __all_sync(kFull, pm1);
    __syncwarp();
    for (int v = lane; v < n; v += 32) {
        const uint2 vi = __ldg(&vinfo[v]);
        const int e1 = (int)vi.x + (int)(vi.y & kDegMask);
        double f = __ldg(&h[v]);
        for (int e = (int)vi.x; e < e1; ++e)
            f = __dadd_rn(f, __dmul_rn((double)(int)sp[__ldg(&col[e])], __ldg(&w[e])));
        de[v] = __dmul_rn((double)(-2 * (int)sp[v]), f);
    }
    __syncwarp();
    return pm1;
}

// The additions of entries `grp` (lanes, in entry order; values in
// scratch) to one slot, in that order.
template <class DE>
__device__ __forceinline__ void add_group(const DE &de, int x, unsigned grp, const double *scratch) {
    if constexpr (DE::kAsyncAdd) {
        while (grp) {
            const int j = __ffs(grp) - 1;
            grp &= grp - 1;
            de.add(x, scratch[j]);
        }
    } else {
        double acc = de.get(x);
        while (grp) {
            const int j = __ffs(grp) - 1;
            grp &= grp - 1;
            acc = __dadd_rn(acc, scratch[j]);
        }
        de.set(x, acc);
    }
}

// cpu_sa.cpp:168-191 for every lane whose bit is set in `fm`.  Lane k of
// the warp holds its variable v, list start `start`, degree `deg` and spin
// `s_old` (valid on flipping lanes).  The flipping variables must be pairwise
// non-adjacent.  Entries are applied lane-parallel in rounds of 32; equal
// targets within a round are summed in entry order by their first lane.
// `scratch` holds 32 doubles followed by 32 ints.  With `own_fresh`, no entry
// of this pass names the lane's own slot, which then still holds `d_own`.
template <class DE>
__device__ __forceinline__ void apply_flips(const Prob &P, DE de, int8_t *sp,
                                            double *scratch, unsigned fm, int v,
                                            int start, int deg, int s_old,
                                            bool may_conflict, unsigned lane,
                                            bool own_fresh = false, double d_own = 0.0) {
    const bool f = (fm >> lane) & 1u;
    const double mult = (double)(int)(int8_t)(4 * s_old);
    int *owner_of_rank = reinterpret_cast<int *>(scratch + 32);
    const int D = P.regular_degree;
    int excl = 0, total;
    if (D) {
        // Equal list lengths: entry t belongs to the (t / D)-th flip.
        if (f) owner_of_rank[__popc(fm & ((1u << lane) - 1u))] = (int)lane;
        total = __popc(fm) * D;
        __syncwarp();
    } else {
        const int my = f ? deg : 0;
        int incl = my;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(kFull, incl, o);
            if ((int)lane >= o) incl += y;
        }
        excl = incl - my;
        total = __shfl_sync(kFull, incl, 31);
    }
    if (!may_conflict && !D) {
        // No two entries name the same slot: each chunk of 96 entries issues
        // all of its delta-energy loads before its stores.
        for (int base = 0; base < total; base += 96) {
            int nb[3];
            double x[3], dv[3];
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const int t = base + 32 * i + (int)lane;
                int k = 0;
#pragma unroll
                for (int step = 16; step > 0; step >>= 1) {
                    const int ex = __shfl_sync(kFull, excl, k + step);
                    if (ex <= t) k += step;
                }
                const int e = __shfl_sync(kFull, start, k) + (t - __shfl_sync(kFull, excl, k));
                const double m_k = __shfl_sync(kFull, mult, k);
                nb[i] = 0;
                x[i] = 0.0;
                if (t < total) {
                    nb[i] = __ldg(&P.col[e]);
                    x[i] = __dmul_rn(__dmul_rn(m_k, __ldg(&P.w[e])), (double)(int)sp[nb[i]]);
                }
            }
            if constexpr (DE::kAsyncAdd) {
#pragma unroll
                for (int i = 0; i < 3; ++i)
                    if (base + 32 * i + (int)lane < total) de.add(nb[i], x[i]);
            } else {
#pragma unroll
                for (int i = 0; i < 3; ++i)
                    if (base + 32 * i + (int)lane < total) dv[i] = de.get(nb[i]);
#pragma unroll
                for (int i = 0; i < 3; ++i)
                    if (base + 32 * i + (int)lane < total) de.set(nb[i], __dadd_rn(dv[i], x[i]));
            }
        }
        __syncwarp();
        total = 0;  // done
    }
    for (int base = 0; base < total; base += 32) {
        const int t = base + (int)lane;
        const bool a = t < total;
        int k, e;
        if (D) {
            const int r = (int)(((uint32_t)t * P.regular_magic) >> 16);  // t / D
            k = a ? owner_of_rank[r] : 0;
            e = __shfl_sync(kFull, v, k) * D + (t - r * D);
        } else {
            // Owner: the last lane whose entry range starts at or before t.
            k = 0;
#pragma unroll
            for (int step = 16; step > 0; step >>= 1) {
                const int ex = __shfl_sync(kFull, excl, k + step);
                if (ex <= t) k += step;
            }
            e = __shfl_sync(kFull, start, k) + (t - __shfl_sync(kFull, excl, k));
        }
        const double m_k = __shfl_sync(kFull, mult, k);
        int nb = -1 - (int)lane;  // distinct per inactive lane
        double x = 0.0;
        if (a) {
            nb = __ldg(&P.col[e]);
            x = __dmul_rn(__dmul_rn(m_k, __ldg(&P.w[e])), (double)(int)sp[nb]);
        }
        const unsigned grp = may_conflict ? __match_any_sync(kFull, nb) : (1u << lane);
        const bool alone = grp == (1u << lane);
        if (a && alone) de.add(nb, x);
        if (may_conflict && __any_sync(kFull, a && !alone)) {
            scratch[lane] = x;
            __syncwarp();
            if (a && !alone && lane == (unsigned)(__ffs(grp) - 1)) {
                add_group(de, nb, grp, scratch);
            }
        }
        __syncwarp();
    }
    if (f) {  // cpu_sa.cpp:189-190, after the variable's own updates
        sp[v] = (int8_t)(-s_old);
        de.set(v, __dmul_rn(own_fresh ? d_own : de.get(v), -1.0));
    }
    __syncwarp();
}

// Adjacency entries t = 32 i + lane (i < kPreGroups) of the accepted flips'
// lists in flip order, loaded before the commit point is known: target,
// coupling and the lane of the entry's flip.
constexpr int kPreGroups = 2;
struct PreEntries {
    int nb[kPreGroups];
    int k[kPreGroups];
    double w[kPreGroups];
};

// Entry t of the flips' lists for equal-length lists (list v at v * D): its
// target, coupling and the lane k of its flip.  `rank_tab[f]` is the lane of
// the f-th flip in variable order.
__device__ __forceinline__ void regular_load(const Prob &P, const int *rank_tab, int p, int t,
                                             int &k, int &nb, double &wt) {
    const int D = P.regular_degree;
    const int r = (int)(((uint32_t)t * P.regular_magic) >> 16);  // t / D
    k = rank_tab[r];
    const int e = (p + k) * D + (t - r * D);
    nb = __ldg(&P.col[e]);
    wt = __ldg(&P.w[e]);
}

// Neighbour updates of the committed flips for equal-length lists.  `mult` is
// each lane's (int8)(4 * s) as a double (cpu_sa.cpp:172), read from the
// entry's owner lane.  With `pre`, the first 32 kPreGroups entries are in `pe`
// (loaded when only the accepted flips were known; the committed flips are a
// prefix of them); the other entries are loaded here.
//
// When no two entries of the pass can name the same slot, the entries go in
// chunks of 32 kPreGroups whose delta-energy loads are all issued before
// their stores, so a chunk waits on memory once.  Otherwise they go in rounds
// of 32, equal targets within a round summed in entry order by their first
// lane, as in apply_flips.
template <class DE>
__device__ __forceinline__ void update_regular(const Prob &P, DE de, const int8_t *sp,
                                               double *scratch, const int *rank_tab,
                                               int nflips, int p, bool pre, const PreEntries &pe,
                                               bool may_conflict, double mult, unsigned lane) {
    const int total = nflips * P.regular_degree;
    if (!may_conflict) {
        for (int base = 0; base < total; base += 32 * kPreGroups) {
            int nb[kPreGroups];
            double x[kPreGroups], dv[kPreGroups];
#pragma unroll
            for (int i = 0; i < kPreGroups; ++i) {
                const int t = base + 32 * i + (int)lane;
                int k = 0, q = 0;
                double wt = 0.0;
                if (pre && base == 0) {
                    k = pe.k[i], q = pe.nb[i], wt = pe.w[i];
                } else if (t < total) {
                    regular_load(P, rank_tab, p, t, k, q, wt);
                }
                const double m_k = __shfl_sync(kFull, mult, k);
                nb[i] = q;
                x[i] = __dmul_rn(__dmul_rn(m_k, wt), (double)(int)sp[q]);
            }
            if constexpr (DE::kAsyncAdd) {
#pragma unroll
                for (int i = 0; i < kPreGroups; ++i)
                    if (base + 32 * i + (int)lane < total) de.add(nb[i], x[i]);
            } else {
#pragma unroll
                for (int i = 0; i < kPreGroups; ++i)
                    if (base + 32 * i + (int)lane < total) dv[i] = de.get(nb[i]);
#pragma unroll
                for (int i = 0; i < kPreGroups; ++i)
                    if (base + 32 * i + (int)lane < total) de.set(nb[i], __dadd_rn(dv[i], x[i]));
            }
        }
        __syncwarp();
        return;
    }
    for (int base = 0; base < total; base += 32) {
        const int t = base + (int)lane;
        const bool a = t < total;
        int k = 0, nb = 0;
        double wt = 0.0;
        if (pre && base == 0) {
            k = pe.k[0], nb = pe.nb[0], wt = pe.w[0];
        } else if (pre && base == 32) {
            k = pe.k[1], nb = pe.nb[1], wt = pe.w[1];
        } else if (a) {
            regular_load(P, rank_tab, p, t, k, nb, wt);
        }
        const double m_k = __shfl_sync(kFull, mult, k);
        double x = 0.0;
        if (a) {
            x = __dmul_rn(__dmul_rn(m_k, wt), (double)(int)sp[nb]);
        } else {
            nb = -1 - (int)lane;  // distinct per inactive lane
        }
        const unsigned grp = __match_any_sync(kFull, nb);
        const bool alone = grp == (1u << lane);
        if (a && alone) de.add(nb, x);
        if (__any_sync(kFull, a && !alone)) {
            scratch[lane] = x;
            __syncwarp();
            if (a && !alone && lane == (unsigned)(__ffs(grp) - 1)) {
                add_group(de, nb, grp, scratch);
            }
        }
        __syncwarp();
    }
}

// cpu_sa.cpp:168-191 for the committed flips `fm` of the window starting at
// p, pulled instead of pushed (problems with dense updates: n <= 128, no
// repeated couplers).  Lane l owns the delta energies of variables l, l + 32,
// l + 64 and l + 96; flip after flip in variable order it adds
// ((int8)(4 s_j) J_jx) s_x to each owned slot x that neighbours j, so every
// slot receives its additions in the reference's order.  Spins are those at
// the start of the pass; the flipped variables' spins and own delta energies
// change last (see sweep_sequential).  `s_cur` is each lane's window spin.
template <class DE>
__device__ __forceinline__ void update_dense(const Prob &P, DE de, int8_t *sp,
                                             unsigned fm, int p, int v, int s_cur,
                                             unsigned lane) {
    const int n = P.n;
    double dx[4], sx[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int x = (int)lane + 32 * i;
        dx[i] = 0.0;
        sx[i] = 0.0;
        if (x < n) {
            dx[i] = de.get(x);
            sx[i] = (double)(int)sp[x];
        }
    }
    unsigned touched = 0u;
    unsigned f = fm;
    while (f) {
        const int j = __ffs(f) - 1;
        f &= f - 1u;
        const double mj = (double)(int)(int8_t)(4 * __shfl_sync(kFull, s_cur, j));
        const int vj = p + j;
        const uint4 bits = __ldg(reinterpret_cast<const uint4 *>(P.dense_bits) + vj);
        const double *__restrict__ row = P.dense_w + (size_t)vj * (size_t)n;
        const uint32_t word[4] = {bits.x, bits.y, bits.z, bits.w};
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            if ((word[i] >> lane) & 1u) {
                const double J = __ldg(&row[(int)lane + 32 * i]);
                dx[i] = __dadd_rn(dx[i], __dmul_rn(__dmul_rn(mj, J), sx[i]));
                touched |= 1u << i;
            }
        }
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
        if ((touched >> i) & 1u) de.set((int)lane + 32 * i, dx[i]);
    __syncwarp();
    if ((fm >> lane) & 1u) {  // cpu_sa.cpp:189-190, after the variable's own updates
        sp[v] = (int8_t)(-s_cur);
        de.set(v, __dmul_rn(de.get(v), -1.0));
    }
    __syncwarp();
}

// One acceptance decision (cpu_sa.cpp:144-166) for a lane that needs a draw:
// the single-precision bounds first, the exact double test inside the band.
// Returns accept in bit 0 and the near-tie flag in bit 1.
template <bool GIBBS>
__device__ __forceinline__ int decide(double d, double beta, uint64_t r) {
    const int fast = GIBBS ? gibbs_fast(__dmul_rn(d, beta), r)
                           : metropolis_fast(__dmul_rn(-d, beta), r);
    if (fast >= 0) return fast;
    return GIBBS ? gibbs_exact(d, beta, r) : metropolis_exact(d, beta, r);
}

// Sequential order (cpu_sa.cpp:132-192) in speculative passes over windows
// of 32 consecutive variables, one per lane.  Every lane decides its variable
// against the delta energies at the start of the pass; the first round
// commits the prefix of the window that ends before the first variable whose
// decision a committed flip could have changed (a later neighbour of an
// accepted flip), so the committed decisions equal the sequential ones.
//
// With `resolve` (problems whose lists name no target twice, reads whose
// spins are all +-1) the pass goes on in further rounds instead of ending
// there.  The flips committed by a round add their contributions
// ((4 s_j) J) s_k (cpu_sa.cpp:172-185) to the delta energies, held in
// registers, of the uncommitted lanes they neighbour, in variable order as the
// reference adds them; those lanes decide again, their draws placed after the
// ones already committed, and the next commit point follows by the same rule.
// Each round commits at least its first lane.  The update phase then applies
// every committed flip's entries to the delta energies in memory in entry
// order with the spins as they were at the start of the pass, and negates the
// flipped variables' own delta energies last: negation is exact and commutes
// with rounding, so a contribution added after the negation in the reference
// (a neighbour that flipped earlier) equals the negated contribution added
// before it.
//
// While a window is processed, the records of the next one are prefetched
// into L1 when the delta energies are on chip or in the band; with resolution
// also the lines of this window's adjacency lists, which the update phase
// reads.
//
// BANDED (kStageBand): the delta energies of variables within band_b of the
// window live in a shared-memory ring of band_w slots (BandDe), the rest in
// the global slot `de_g`.  After each pass the band slides by the committed
// count: the slots leaving it are written back and the ones entering are
// fetched asynchronously.  band_w >= 2 band_b + 128 keeps the slots fetched
// by a slide at least four passes ahead of the window, so every pass waits
// only for the slides before the last one (cp.async.wait_group 1) before its
// decisions read the window; an update through a coupler longer than band_b
// can reach the last slide's slots, so the update phase waits for all of
// them.  At every sweep the band is written back and reloaded from the start.
template <bool GIBBS, bool DENSE_OK, int STAGE>
__device__ __forceinline__ void sweep_sequential(const Prob &P, double *de_g,
                                                 int8_t *sp, double *scratch,
                                                 uint64_t *ring, RingState &rs,
                                                 unsigned lane, bool resolve,
                                                 double *band, int band_w, int band_b) {
    constexpr bool BANDED = STAGE == kStageBand;
    const int n = P.n;
    const int D = P.regular_degree;
    const unsigned lt_mask = (1u << lane) - 1u;
    int *rank_tab = reinterpret_cast<int *>(scratch + 32);
    typename DeFor<STAGE>::T de;
    bool band_live = false;
    if constexpr (BANDED)
        de = BandDe{de_g, band, 0, (unsigned)band_w};
    else
        de.p = de_g;
    for (int b = 0; b < reload(P.pd->num_betas); ++b) {
        const double beta = __ldg(&reload(P.pd->betas)[b]);
        const double thr = __ldg(&reload(P.pd->thresholds)[b]);
        for (int sw = 0; sw < reload(P.pd->sweeps_per_beta); ++sw) {
            SweepCount cnt;
            if constexpr (BANDED) {
                if (band_w) {  // write the band back, reload it at the start
                    cp_async_wait<0>();
                    __syncwarp();
                    const unsigned mask = (unsigned)band_w - 1u;
                    if (band_live) {
                        for (int i = (int)lane; i < band_w; i += 32) {
                            const int x = de.lo + i;
                            if (x >= 0 && x < n) de_g[x] = band[(unsigned)x & mask];
                        }
                        __syncwarp();
                    }
                    de.lo = -band_b;
                    const int top = min(n, band_w - band_b);
                    for (int x = (int)lane; x < top; x += 32) band[(unsigned)x & mask] = de_g[x];
                    __syncwarp();
                    band_live = true;
                }
            }
            int p = 0;
            while (p < n) {
                if constexpr (BANDED) {
                    if (band_w) {  // the slides of all but the last pass have landed
                        cp_async_wait<1>();
                        __syncwarp();
                    }
                }
                ring_refill(ring, rs, lane);
                const int L = min(32, n - p);
                const int v = p + (int)lane;
                const bool act = (int)lane < L;
                double d = 0.0;
                int dist = (int)kDistCap;
                uint32_t shr = 0u;
                uint2 vi = make_uint2(0u, 0u);
                uint2 bk = make_uint2(0u, 0u);
                int s_cur = 0;
                if (act) {
                    d = de.get(v);
                    dist = __ldg(&P.dist[v]);
                    shr = __ldg(&P.share[v]);
                    if (!D) vi = __ldg(&P.vinfo[v]);
                    if (resolve) bk = __ldg(&P.back[v]);
                    s_cur = (int)sp[v];
                }
                // The nearest back neighbour's coupling (stored last), loaded
                // ahead: on lattices and chains it is the one the rounds need.
                int o_near = 0;
                double bw_near = 0.0;
                if (resolve && bk.x) {
                    o_near = __ffs(bk.x) - 1;
                    bw_near = __ldg(&P.bw[bk.y + (uint32_t)__popc(bk.x) - 1u]);
                }
                if (act) {
                    // The next window starts at p + c <= p + 32 and ends
                    // before p + c + 32, so the lines of [v + 32] are the
                    // ones it may need beyond this window's.
                    const int vn = v + 32;
                    // (Not with global slots: there the prefetches measured
                    // slower than the plain loads.)
                    if (vn < n && !DeFor<STAGE>::T::kAsyncAdd) {
                        prefetch_l1(P.dist + vn);
                        prefetch_l1(P.share + vn);
                        if (!D) prefetch_l1(P.vinfo + vn);
                        if (resolve) prefetch_l1(P.back + vn);
                    }
                    if (resolve) {  // the update phase's lists (no early load with resolution)
                        const uint32_t e0 = D ? (uint32_t)v * (uint32_t)D : vi.x;
                        prefetch_l1(P.col + e0);
                        prefetch_l1(P.w + e0);
                    }
                }
                const bool consider = act && !(d >= thr);  // cpu_sa.cpp:140
                const bool need = GIBBS ? consider : (consider && !(d <= 0.0));
                const unsigned nm = __ballot_sync(kFull, need);
                bool acc = GIBBS ? false : consider;  // Metropolis: d <= 0 accepts
                bool near = false;
                if (need) {
                    const uint64_t r = ring[(rs.q + (uint32_t)__popc(nm & lt_mask)) & (kRing - 1)];
                    const int x = decide<GIBBS>(d, beta, r);
                    acc = (x & 1) != 0;
                    near = (x & 2) != 0;
                }
                const unsigned am = __ballot_sync(kFull, acc);
                // Equal-length lists: start loading the accepted flips'
                // adjacency before the commit point is known (not with
                // resolution, whose later rounds change the accepted set).
                const bool pre = !resolve;
                const double mult = (double)(int)(int8_t)(4 * s_cur);
                PreEntries pe;
#pragma unroll
                for (int i = 0; i < kPreGroups; ++i) pe.nb[i] = 0, pe.k[i] = 0, pe.w[i] = 0.0;
                if (D && am && pre) {
                    if (acc) rank_tab[__popc(am & lt_mask)] = (int)lane;
                    __syncwarp();
                    const int pre_n = min(__popc(am) * D, 32 * kPreGroups);
#pragma unroll
                    for (int i = 0; i < kPreGroups; ++i) {
                        const int t = (int)lane + 32 * i;
                        if (t < pre_n) regular_load(P, rank_tab, p, t, pe.k[i], pe.nb[i], pe.w[i]);
                    }
                }
                const int bound = acc ? (int)lane + dist : 32;
                int c = min(__reduce_min_sync(kFull, bound), L);
                unsigned done = c >= 32 ? kFull : ((1u << c) - 1u);
                uint32_t used = (uint32_t)__popc(nm & done);
                unsigned fm = am & done;
                unsigned nearm = __ballot_sync(kFull, near) & done;
                if (resolve && c < L) {
                    // Lanes j < lane whose variables neighbour this lane's.
                    const unsigned back_lanes = __brev(bk.x) >> (31u - lane);
                    const unsigned smask = __ballot_sync(kFull, s_cur > 0);
                    const double sk = (double)s_cur;
                    unsigned newf = fm;
                    // Each lane keeps the flags of its latest decision; a
                    // committed lane's are final, so the ballots of a round
                    // cover the committed lanes too (its draw position counts
                    // the committed draws before it).
                    bool need_l = need, acc_l = acc;
                    unsigned nm_all;
                    do {
                        const bool live = act && (int)lane >= c;
                        unsigned rel = live ? back_lanes & newf : 0u;
                        while (rel) {
                            const int j = __ffs(rel) - 1;
                            rel &= rel - 1u;
                            const int o = (int)lane - j;
                            double wj = bw_near;
                            if (o != o_near) {
                                // Offsets are stored descending: o's rank is
                                // the number of larger offsets.
                                wj = __ldg(&P.bw[bk.y + (uint32_t)__popc((bk.x >> o) >> 1)]);
                            }
                            const double mj = ((smask >> j) & 1u) ? 4.0 : -4.0;
                            d = __dadd_rn(d, __dmul_rn(__dmul_rn(mj, wj), sk));
                        }
                        if (live) {
                            const bool cons2 = !(d >= thr);
                            need_l = GIBBS ? cons2 : (cons2 && !(d <= 0.0));
                            acc_l = GIBBS ? false : cons2;
                            near = false;
                        }
                        nm_all = __ballot_sync(kFull, need_l);
                        if (live && need_l) {
                            const uint64_t r =
                                ring[(rs.q + (uint32_t)__popc(nm_all & lt_mask)) & (kRing - 1)];
                            const int x = decide<GIBBS>(d, beta, r);
                            acc_l = (x & 1) != 0;
                            near = (x & 2) != 0;
                        }
                        const unsigned am_all = __ballot_sync(kFull, acc_l);
                        const int bound2 = (live && acc_l) ? (int)lane + dist : 32;
                        c = min(__reduce_min_sync(kFull, bound2), L);
                        const unsigned upto = c >= 32 ? kFull : ((1u << c) - 1u);
                        newf = am_all & upto & ~done;
                        fm = am_all & upto;
                        done = upto;
                    } while (c < L);
                    used = (uint32_t)__popc(nm_all & done);
                    nearm = __ballot_sync(kFull, near) & done;
                }
                rs.q += used;
                cnt.pass((unsigned)__popc(fm), (unsigned)__popc(nearm));
                if constexpr (BANDED) {
                    // The slots the last slide fetched lie at the far end of
                    // the band, which only an update through a coupler longer
                    // than band_b can reach: they land before the update phase.
                    if (band_w && fm) {
                        cp_async_wait<0>();
                        __syncwarp();
                    }
                }
                if (fm && DENSE_OK && P.dense) {
                    update_dense(P, de, sp, fm, p, v, s_cur, lane);
                } else if (fm) {
                    // A slot can receive two additions only through a repeated
                    // target in one list or a neighbour common to two flips.
                    const unsigned later = lane < 31 ? fm >> (lane + 1) : 0u;
                    const bool f = (fm >> lane) & 1u;
                    const bool may_conflict =
                        __any_sync(kFull, f && ((shr & 1u) || ((shr >> 1) & later)));
                    // Without resolution the committed flips are pairwise
                    // non-adjacent, so a flip's own slot receives an addition
                    // in this pass only from a repeated target in its own
                    // list; otherwise it still holds the window value d and
                    // the negation needs no load.
                    const bool own_fresh = !resolve && !(shr & 1u);
                    if (D) {
                        if (!pre) {
                            if (f) rank_tab[__popc(fm & lt_mask)] = (int)lane;
                            __syncwarp();
                        }
                        update_regular(P, de, sp, scratch, rank_tab, __popc(fm), p, pre, pe,
                                       may_conflict, mult, lane);
                        if (f) {  // cpu_sa.cpp:189-190, after the variable's own updates
                            sp[v] = (int8_t)(-s_cur);
                            de.set(v, __dmul_rn(own_fresh ? d : de.get(v), -1.0));
                        }
                        __syncwarp();
                    } else {
                        apply_flips(P, de, sp, scratch, fm, v, (int)vi.x,
                                    (int)(vi.y & kDegMask), s_cur, may_conflict, lane, own_fresh,
                                    d);
                    }
                }
                if constexpr (BANDED) {
                    if (band_w) {  // slide the band by c
                        __syncwarp();
                        if ((int)lane < c) {
                            const int xo = p - band_b + (int)lane;  // < p: band_b >= 32
                            const unsigned slot = (unsigned)xo & ((unsigned)band_w - 1u);
                            if (xo >= 0) de_g[xo] = band[slot];
                            const int xn = xo + band_w;
                            if (xn < n) cp_async8(&band[slot], &de_g[xn]);
                        }
                        cp_async_commit();
                        __syncwarp();
                    }
                }
                p += c;
                if constexpr (BANDED) de.lo = p - band_b;
            }
            cnt.flush(ring, lane);
        }
    }
    if constexpr (BANDED) {
        if (band_w) {  // nothing of this read may land after it
            cp_async_wait<0>();
            __syncwarp();
        }
    }
}

// Random order (cpu_sa.cpp:134-139) in speculative windows of the RNG
// stream.  Each attempt draws its variable as rand % n and, when it needs one,
// its acceptance draw right after it.  Lane l takes stream position q + l as
// the variable draw of a possible attempt and q + l + 1 as that attempt's
// acceptance draw, and decides it against the delta energies at the start of
// the pass.  The attempts actually made form a chain: lane 0, then each
// chain lane's successor at l + 1, or l + 2 when l drew for its acceptance.
// A chain lane's decision stands unless an earlier accepted flip of the
// window touched its variable (flipped it or a neighbour of it); the window
// commits the chain up to the first such lane.  Touched variables are marked
// in a per-warp bitmap (`touch`, n bits, clear between passes).  Committed
// flips are pairwise distinct and non-adjacent, so their neighbour updates
// are applied together, equal targets summed in entry order.
template <bool GIBBS, class DE>
__device__ __forceinline__ void sweep_random(const Prob &P, DE de,
                                             int8_t *sp, double *scratch,
                                             uint64_t *ring, RingState &rs,
                                             unsigned lane, uint32_t *touch) {
    const int n = P.n;
    const int D = P.regular_degree;
    for (int b = 0; b < reload(P.pd->num_betas); ++b) {
        const double beta = __ldg(&reload(P.pd->betas)[b]);
        const double thr = __ldg(&reload(P.pd->thresholds)[b]);
        for (int sw = 0; sw < reload(P.pd->sweeps_per_beta); ++sw) {
            SweepCount cnt;
            int rem = n;  // attempts left in this sweep
            while (rem > 0) {
                ring_refill(ring, rs, lane);
                const uint64_t rv = ring[(rs.q + lane) & (kRing - 1)];
                const int var = (int)(rv % (uint64_t)n);  // cpu_sa.cpp:135-136
                const double d = de.get(var);
                const bool cons = !(d >= thr);            // cpu_sa.cpp:140
                const bool need = GIBBS ? cons : (cons && !(d <= 0.0));
                const unsigned N = __ballot_sync(kFull, need);
                // Chain lanes: l is on the chain unless l - 1 is a chain lane
                // that drew.  Inside a run of drawing lanes starting at a, the
                // chain takes a, a + 2, ...; elsewhere every lane.
                bool on = true;
                if (lane > 0 && ((N >> (lane - 1)) & 1u)) {
                    const unsigned starts = N & ~(N << 1);
                    const unsigned below = starts & ((2u << (lane - 1)) - 1u);
                    const int a = 31 - __clz(below);
                    on = (((int)lane - a) & 1) == 0;
                }
                unsigned C = __ballot_sync(kFull, on);
                if (__popc(C) > rem) {  // the sweep ends inside the window
                    unsigned t = C;
                    for (int i = 0; i < rem; ++i) t &= t - 1u;
                    C &= ~t;
                }
                const bool chain = (C >> lane) & 1u;
                bool acc = false, near = false;
                if (chain) {
                    acc = GIBBS ? false : cons;  // Metropolis: d <= 0 accepts
                    if (need) {
                        const uint64_t r = ring[(rs.q + lane + 1u) & (kRing - 1)];
                        const int x = decide<GIBBS>(d, beta, r);
                        acc = (x & 1) != 0;
                        near = (x & 2) != 0;
                    }
                }
                const unsigned A = __ballot_sync(kFull, acc);
                // Commit point: the first chain lane whose variable an earlier
                // accepted flip touched.  Accepted lanes are marked in order.
                int c = 32;
                unsigned todo = A, marked = 0u;
                while (todo) {
                    const int j = __ffs(todo) - 1;
                    if (j >= c) break;
                    todo &= todo - 1u;
                    marked |= 1u << j;
                    const int vj = __shfl_sync(kFull, var, j);
                    const uint2 vi = D ? make_uint2((uint32_t)vj * (uint32_t)D, (uint32_t)D)
                                       : __ldg(&P.vinfo[vj]);
                    const int deg = (int)(vi.y & kDegMask);
                    for (int t = (int)lane; t < deg; t += 32) {
                        const int x = __ldg(&P.col[vi.x + (uint32_t)t]);
                        atomicOr(&touch[x >> 5], 1u << (x & 31));
                    }
                    if (lane == 0) atomicOr(&touch[vj >> 5], 1u << (vj & 31));
                    __syncwarp();
                    const bool hit = chain && (int)lane > j && ((touch[var >> 5] >> (var & 31)) & 1u);
                    const unsigned H = __ballot_sync(kFull, hit);
                    if (H) c = min(c, __ffs(H) - 1);
                }
                if (marked) {  // clear the marked words for the next pass
                    __syncwarp();
                    unsigned m = marked;
                    while (m) {
                        const int j = __ffs(m) - 1;
                        m &= m - 1u;
                        const int vj = __shfl_sync(kFull, var, j);
                        const uint2 vi = D ? make_uint2((uint32_t)vj * (uint32_t)D, (uint32_t)D)
                                           : __ldg(&P.vinfo[vj]);
                        const int deg = (int)(vi.y & kDegMask);
                        for (int t = (int)lane; t < deg; t += 32)
                            touch[__ldg(&P.col[vi.x + (uint32_t)t]) >> 5] = 0u;
                        if (lane == 0) touch[vj >> 5] = 0u;
                    }
                    __syncwarp();
                }
                const unsigned cm = C & (c >= 32 ? kFull : ((1u << c) - 1u));
                const int last = 31 - __clz(cm);  // lane 0 is always committed
                rs.q += (uint32_t)(last + 1) + ((N >> last) & 1u);
                rem -= __popc(cm);
                const unsigned fm = A & cm;
                cnt.pass((unsigned)__popc(fm), (unsigned)__popc(__ballot_sync(kFull, near) & cm));
                if (fm) {
                    const int s_old = (int)sp[var];
                    const uint2 vi = D ? make_uint2((uint32_t)var * (uint32_t)D, (uint32_t)D)
                                       : __ldg(&P.vinfo[var]);
                    __syncwarp();
                    apply_flips(P, de, sp, scratch, fm, var, (int)vi.x, (int)(vi.y & kDegMask),
                                s_old, true, lane);
                }
            }
            cnt.flush(ring, lane);
        }
    }
}

// cpu_sa.cpp:210-227.  Terms are formed lane-parallel (each an exact
// rounding of the same operands); the running sum is strictly sequential.
__device__ __forceinline__ double state_energy(const ProblemDev *PD, const int8_t *sp,
                                               unsigned lane) {
    const int n = PD->n;
    const int64_t m = PD->m;
    const double *__restrict__ h = PD->h;
    const int32_t *__restrict__ cu = PD->cu;
    const int32_t *__restrict__ cv = PD->cv;
    const double *__restrict__ cw = PD->cw;
    double e = 0.0;
    for (int base = 0; base < n; base += 32) {
        const int v = base + (int)lane;
        const double t = v < n ? __dmul_rn((double)(int)sp[v], __ldg(&h[v])) : 0.0;
        const int cnt = min(32, n - base);
        for (int j = 0; j < cnt; ++j) e = __dadd_rn(e, __shfl_sync(kFull, t, j));
    }
    for (int64_t base = 0; base < m; base += 32) {
        const int64_t c = base + lane;
        double t = 0.0;
        if (c < m)
            t = __dmul_rn(__dmul_rn((double)(int)sp[__ldg(&cu[c])], __ldg(&cw[c])),
                          (double)(int)sp[__ldg(&cv[c])]);
        const int cnt = (int)min((int64_t)32, m - base);
        for (int j = 0; j < cnt; ++j) e = __dadd_rn(e, __shfl_sync(kFull, t, j));
    }
    return e;
}

template <bool GIBBS, bool RANDOM_ORDER, bool RESOLVE, int STAGE>
__device__ __forceinline__ void anneal_read(const ProblemDev *PD, const int8_t *src,
                                            int8_t *dst, double *energy_out,
                                            double *de, int8_t *sp,
                                            double *scratch, uint64_t *ring,
                                            RingState &rs, unsigned lane, uint32_t *touch,
                                            double *band, int band_cap) {
    const bool pm1 = load_state(PD, src, de, sp, lane);
    {
        const Prob P = load_prob(PD);
        if constexpr (RANDOM_ORDER) {
            static_assert(STAGE != kStageBand, "the band follows a sequential window");
            typename DeFor<STAGE>::T acc;
            acc.p = de;
            sweep_random<GIBBS>(P, acc, sp, scratch, ring, rs, lane, touch);
        } else {
            // A problem whose band does not fit the launch's ring keeps all of
            // its delta energies in the global slot.
            const int bw = (STAGE == kStageBand && PD->band_w > 0 && PD->band_w <= band_cap)
                               ? PD->band_w
                               : 0;
            sweep_sequential<GIBBS, RESOLVE, STAGE>(P, de, sp, scratch, ring, rs, lane,
                                                    RESOLVE && pm1, band, bw, PD->band_b);
        }
    }
    __syncwarp();
    const double e = state_energy(PD, sp, lane);
    const int n = PD->n;
    for (int v = lane; v < n; v += 32) dst[v] = sp[v];
    if (lane == 0) *energy_out = e;
    __syncwarp();
}

}  // namespace b200sa
