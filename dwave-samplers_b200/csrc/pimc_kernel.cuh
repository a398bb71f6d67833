// Path-integral Monte Carlo annealing (the reference's SQA localPIMC,
// dwave/samplers/sqa/src/localPIMC.cpp) on the GPU.  Included by
// sa_launch.cu next to the annealing kernels.
//
// One thread per sample.  An update draws a data-dependent number of random
// numbers (break proposals, one Gibbs draw per domain) from one mt19937
// stream and merges variable-length break lists, so a sample is one
// sequential chain; many samples run side by side.  Every sample keeps its
// world lines in global memory: the first Trotter slice (int8 spins), the
// number of breaks of each variable and their positions (cap_breaks slots per
// variable, increasing).  Every slot (thread) keeps its mt19937 state and a
// scratch area (proposals, interfaces, domain fields, chain labels).
//
// Arithmetic follows localPIMC.cpp operation for operation:
//   run (:126-157)              Hd sets Gamma, Hp sets invTemp per schedule step;
//                               sweeps_per_beta * n updates of uniformly drawn
//                               qubits (or chains) per step
//   qubitUpdate (:361-393), chainUpdate (:395-464), makeDomainGraph (:474-541)
//   addHToEffectiveField (:277-295), addJToEffectiveField (:297-359)
//   makeBreakProposals (:543-555), GibbsSamplePM1, pNotJoin (:568-576)
//   get_state_energy (:59-75)
// and std::mt19937 with libstdc++'s uniform_int_distribution (Lemire's
// method on the 64-bit product) and generate_canonical<double, 53>.
//
// Where the reference calls libm (log, tanh, exp) this calls CUDA's; every
// decision they feed is checked against a relative band of 2^-48 around its
// threshold and counted as a near tie (0 expected; the host reports them).
#pragma once
#include "sa_kernel.cuh"

namespace b200sa {

constexpr int kPimcSlices = 65536;  // numTrotterSlices, localPIMC.h:88

// mt19937 (Matsumoto & Nishimura 1998), regenerated one word per draw: word
// i is replaced by its successor from words i, i + 1 and i + 397 (mod 624) just
// before it is output.  Regenerating in index order is what the block
// regeneration of all 624 words does, so the stream is the same; the cost is
// the same for every draw, so threads of a warp never wait on one thread's
// 624-word burst.
struct PimcRng {
    uint32_t *mt;
    int idx;       // next word to regenerate and output
    uint32_t cur;  // mt[idx], not yet regenerated

    __device__ void seed(uint32_t s) {
        uint32_t x = s;
        mt[0] = x;
        for (int i = 1; i < kMtWords; ++i) {
            x = 1812433253u * (x ^ (x >> 30)) + (uint32_t)i;
            mt[i] = x;
        }
        idx = 0;
        cur = s;
    }
    __device__ __forceinline__ uint32_t next() {
        const int i1 = idx == kMtWords - 1 ? 0 : idx + 1;
        const int im = idx < kMtWords - 397 ? idx + 397 : idx - (kMtWords - 397);
        const uint32_t b = mt[i1];
        const uint32_t t = (cur & 0x80000000u) | (b & 0x7fffffffu);
        uint32_t y = mt[im] ^ (t >> 1) ^ ((t & 1u) ? 0x9908b0dfu : 0u);
        mt[idx] = y;
        idx = i1;
        cur = b;
        y ^= y >> 11;
        y ^= (y << 7) & 0x9d2c5680u;
        y ^= (y << 15) & 0xefc60000u;
        y ^= y >> 18;
        return y;
    }
    // generate_canonical<double, 53>: (d1 + d2 * 2^32) / 2^64, below 1.
    __device__ __forceinline__ double canonical() {
        const double lo = __uint2double_rn(next());
        const double hi = __uint2double_rn(next());
        const double r = __ddiv_rn(__dadd_rn(lo, __dmul_rn(hi, 4294967296.0)), kTwo64);
        return r >= 1.0 ? 0x1.fffffffffffffp-1 : r;  // nextafter(1, 0)
    }
    // uniform_int_distribution<int>(0, range - 1).
    __device__ __forceinline__ int below(uint32_t range) {
        uint64_t prod = (uint64_t)next() * range;
        uint32_t low = (uint32_t)prod;
        if (low < range) {
            const uint32_t threshold = (0u - range) % range;
            while (low < threshold) {
                prod = (uint64_t)next() * range;
                low = (uint32_t)prod;
            }
        }
        return (int)(prod >> 32);
    }
};

// The per-thread view of one sample's world lines.
struct PimcWorld {
    int8_t *s;        // [n]
    int32_t *cnt;     // [n]
    int32_t *brk;     // [n][cap]
    int cap;
    double beta, gamma;
    unsigned near;
    bool overflow;

    __device__ const int32_t *list(int v) const { return brk + (int64_t)v * cap; }
    __device__ int32_t *list(int v) { return brk + (int64_t)v * cap; }
};

// makeBreakProposals: positions with exponential gaps of scale slices / Gamma.
__device__ int pimc_proposals(PimcRng &g, PimcWorld &W, int32_t *out, int cap) {
    const double neg_scale = -__ddiv_rn((double)kPimcSlices, W.gamma);
    int k = 0;
    double x = __dmul_rn(neg_scale, log(g.canonical()));
    double position = x;
    for (;;) {
        // int(position) and the bound both switch at integers.
        if (position < (double)(kPimcSlices + 1) && isfinite(position))
            W.near += fabs(position - rint(position)) <= fmax(fabs(x), 1.0) * kTieRel;
        if (!(position < (double)kPimcSlices)) break;
        if (k == cap) {
            W.overflow = true;
            return k;
        }
        out[k] = (int)position;
        x = __dmul_rn(neg_scale, log(g.canonical()));
        position = __dadd_rn(__dadd_rn(x, (double)out[k]), 1.0);
        ++k;
    }
    return k;
}

// std::merge(a, b): on equal values the element of a comes first.
__device__ int pimc_merge(const int32_t *a, int na, const int32_t *b, int nb, int32_t *out) {
    int i = 0, j = 0, k = 0;
    while (i < na && j < nb) out[k++] = b[j] < a[i] ? b[j++] : a[i++];
    while (i < na) out[k++] = a[i++];
    while (j < nb) out[k++] = b[j++];
    return k;
}

// Interfaces of qubit q: proposals merged with its breaks, or the single
// book-keeping value when there is at most one of them together.
__device__ int pimc_interfaces(PimcRng &g, PimcWorld &W, int q, int32_t *props, int cap_props,
                               int32_t *itf) {
    const int np = pimc_proposals(g, W, props, cap_props);
    const int nb = W.cnt[q];
    if (np + nb > 1) return pimc_merge(props, np, W.list(q), nb, itf);
    itf[0] = kPimcSlices;
    return 1;
}

// addHToEffectiveField; lab maps a domain to its accumulator (null: itself).
__device__ void pimc_add_h(double *eff, const int32_t *lab, const int32_t *itf, int nd,
                           double H) {
    H = __ddiv_rn(H, (double)kPimcSlices);
    const int d0 = lab ? lab[0] : 0;
    eff[d0] = __dadd_rn(eff[d0], __dmul_rn((double)(kPimcSlices + itf[0] - itf[nd - 1]), H));
    for (int i = 1; i < nd; ++i) {
        const int d = lab ? lab[i] : i;
        eff[d] = __dadd_rn(eff[d], __dmul_rn((double)(itf[i] - itf[i - 1]), H));
    }
}

// addJToEffectiveField: the neighbour's spin, flipped at each of its breaks,
// over the domains of this qubit.  The merged list (neighbour first on equal
// values) is walked without being stored.
__device__ void pimc_add_j(double *eff, const int32_t *lab, const int32_t *itf, int nd,
                           const int32_t *nbk, int nn, double Js) {
    Js = __ddiv_rn(Js, (double)kPimcSlices);
    int i = 0, j = 0;  // cursors into nbk and itf
    auto next = [&]() { return (i >= nn || (j < nd && itf[j] < nbk[i])) ? itf[j++] : nbk[i++]; };
    const int L = nn + nd;
    const int front = nn ? min(nbk[0], itf[0]) : itf[0];
    const int back = nn ? max(nbk[nn - 1], itf[nd - 1]) : itf[nd - 1];
    const int d0 = lab ? lab[0] : 0;
    eff[d0] = __dadd_rn(eff[d0], __dmul_rn((double)(kPimcSlices + front - back), Js));
    int cur = next();
    int k = 0, oi = 0;
    for (; k + 1 < L; ++k) {
        if (cur == itf[oi]) {
            if (++oi == nd) break;
        } else {
            Js = -Js;
        }
        const int nxt = next();
        const int d = lab ? lab[oi] : oi;
        eff[d] = __dadd_rn(eff[d], __dmul_rn((double)(nxt - cur), Js));
        cur = nxt;
    }
    for (; k + 1 < L; ++k) {
        const int nxt = next();
        eff[d0] = __dadd_rn(eff[d0], __dmul_rn((double)(nxt - cur), Js));
        Js = -Js;
        cur = nxt;
    }
}

// Adds h and every neighbour's world line of qubit q to the domain fields,
// neighbours in adjacency order.  The spin, break count and coupling of up
// to four neighbours are loaded before any field is written, so those loads
// overlap instead of waiting behind the previous neighbour's stores.
__device__ void pimc_fields(const PimcArgs &A, const PimcWorld &W, int q, double *eff,
                            const int32_t *lab, const int32_t *itf, int nd) {
    pimc_add_h(eff, lab, itf, nd, __ldg(&A.h[q]));
    const uint2 vi = __ldg(&A.vinfo[q]);
    const unsigned end = vi.x + vi.y;
    for (unsigned k0 = vi.x; k0 < end; k0 += 4) {
        int nb[4], cnt[4];
        double js[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) nb[j] = k0 + j < end ? __ldg(&A.col[k0 + j]) : 0;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            if (k0 + j < end) {
                cnt[j] = W.cnt[nb[j]];
                js[j] = __dmul_rn((double)W.s[nb[j]], __ldg(&A.w[k0 + j]));
            }
        }
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if (k0 + j < end) pimc_add_j(eff, lab, itf, nd, W.list(nb[j]), cnt[j], js[j]);
    }
}

__device__ __forceinline__ int pimc_gibbs(PimcRng &g, PimcWorld &W, double field) {
    const double thr = __dadd_rn(__dmul_rn(g.canonical(), 2.0), -1.0);  // uniform(-1, 1)
    const double t = tanh(__dmul_rn(W.beta, field));
    W.near += fabs(t - thr) <= fabs(t) * kTieRel;
    return t > thr ? -1 : 1;
}

// pNotJoin(overlaps) < uniform(0, 1)
__device__ __forceinline__ bool pimc_join(PimcRng &g, PimcWorld &W, double jchain, int overlaps) {
    const double p = exp(__ddiv_rn(
        __dmul_rn(__dmul_rn(__dmul_rn(2.0, jchain), (double)overlaps), W.beta),
        (double)kPimcSlices));
    const double c = g.canonical();
    W.near += fabs(p - c) <= p * kTieRel;
    return p < c;
}

// Rewrites the breaks of qubit q from its interfaces and the spins of its
// domains; returns false (overflow) when they do not fit.
template <typename SPIN>
__device__ bool pimc_store(PimcWorld &W, int q, const int32_t *itf, int nd, SPIN spin) {
    const int first = spin(0);
    W.s[q] = (int8_t)first;
    int32_t *out = W.list(q);
    int c = 0, sv = first;
    for (int d = 1; d < nd; ++d) {
        if (sv * spin(d) != 1) {
            sv = -sv;
            if (c == W.cap) return false;
            out[c++] = itf[d - 1];
        }
    }
    if (sv != first) {
        if (c == W.cap) return false;
        out[c++] = itf[nd - 1];
    }
    W.cnt[q] = c;
    return true;
}

// qubitUpdate (localPIMC.cpp:361-393).  Gibbs draws go domain by domain in
// order, so drawing them all before rewriting the breaks keeps the stream.
__device__ void pimc_qubit_update(const PimcArgs &A, PimcRng &g, PimcWorld &W, int sp,
                                  int32_t *props, int32_t *itf, int32_t *sv, double *eff) {
    const int nd = pimc_interfaces(g, W, sp, props, A.cap_props, itf);
    if (W.overflow) return;
    for (int i = 0; i < nd; ++i) eff[i] = 0.0;
    pimc_fields(A, W, sp, eff, nullptr, itf, nd);
    for (int d = 0; d < nd; ++d) sv[d] = pimc_gibbs(g, W, eff[d]);
    if (!pimc_store(W, sp, itf, nd, [&](int d) { return sv[d]; })) W.overflow = true;
}

__device__ __forceinline__ int pimc_find(int32_t *parent, int x) {
    while (parent[x] != x) {
        parent[x] = parent[parent[x]];
        x = parent[x];
    }
    return x;
}

// Parents always point to smaller indices, so pimc_find ends.
__device__ __forceinline__ void pimc_union(int32_t *parent, int a, int b) {
    a = pimc_find(parent, a);
    b = pimc_find(parent, b);
    if (a != b) parent[max(a, b)] = min(a, b);
}

// makeDomainGraph (localPIMC.cpp:474-541) for chain qubits c and c + 1:
// joins go straight into a union-find forest over the domains.
__device__ void pimc_domain_graph(const PimcArgs &A, PimcRng &g, PimcWorld &W, int sp, int c,
                                  const int32_t *itfA, int nA, int z, const int32_t *itfB,
                                  int nB, int f, int32_t *pair, int32_t *parent) {
    const int q = sp * A.qpc + c;
    int s0s1 = (int)W.s[q] * (int)W.s[q + 1];
    int L = pimc_merge(itfA, nA, itfB, nB, pair);
    if (pair[0] == kPimcSlices) {
        if (s0s1 == 1 && pimc_join(g, W, A.jchain, kPimcSlices)) pimc_union(parent, z, f);
        return;
    }
    if (pair[L - 1] == kPimcSlices) --L;
    if (s0s1 == 1 && pimc_join(g, W, A.jchain, kPimcSlices - pair[L - 1] + pair[0]))
        pimc_union(parent, z, f);
    const int32_t *b0 = W.list(q), *b1 = W.list(q + 1);
    const int n0 = W.cnt[q], n1 = W.cnt[q + 1];
    int p0 = 0, e0 = 0, p1 = 0, e1 = 0;
    bool valid0 = itfA[0] != kPimcSlices;
    for (int i = 1; i < L; ++i) {
        if (valid0 && pair[i - 1] == itfA[p0]) {
            if (nA == ++p0) {
                valid0 = false;
                p0 = 0;
            }
            if (n0 > e0 && pair[i - 1] == b0[e0]) {
                s0s1 = -s0s1;
                ++e0;
            }
        } else {
            if (nB == ++p1) p1 = 0;
            if (n1 > e1 && pair[i - 1] == b1[e1]) {
                s0s1 = -s0s1;
                ++e1;
            }
        }
        if (s0s1 == 1 && pimc_join(g, W, A.jchain, pair[i] - pair[i - 1]))
            pimc_union(parent, z + p0, f + p1);
    }
}

// chainUpdate (localPIMC.cpp:395-464).  Components are numbered in order of
// their smallest domain, as the reference's depth-first labelling from roots
// 0, 1, ... numbers them.  Scratch: itf [Q][C], off [Q + 1], lab / parent /
// sv [Q * C], pair [2C], eff [Q * C].
__device__ void pimc_chain_update(const PimcArgs &A, PimcRng &g, PimcWorld &W, int sp,
                                  int32_t *props, int32_t *itf, int32_t *off, int32_t *lab,
                                  int32_t *parent, int32_t *sv, int32_t *pair, double *eff) {
    const int Q = A.qpc;
    const int C = A.cap_props + A.cap_breaks;
    int total = 0;
    for (int c = 0; c < Q; ++c) {
        const int nd = pimc_interfaces(g, W, Q * sp + c, props, A.cap_props, itf + c * C);
        if (W.overflow) return;
        off[c] = total;
        total += nd;
    }
    off[Q] = total;
    for (int d = 0; d < total; ++d) parent[d] = d;
    for (int c = 0; c + 1 < Q; ++c)
        pimc_domain_graph(A, g, W, sp, c, itf + c * C, off[c + 1] - off[c], off[c],
                          itf + (c + 1) * C, off[c + 2] - off[c + 1], off[c + 1], pair, parent);
    int ncomp = 0;
    for (int d = 0; d < total; ++d) sv[d] = -1;  // label of each root
    for (int d = 0; d < total; ++d) {
        const int r = pimc_find(parent, d);
        if (sv[r] < 0) sv[r] = ncomp++;
        lab[d] = sv[r];
    }
    for (int k = 0; k < ncomp; ++k) eff[k] = 0.0;
    for (int c = 0; c < Q; ++c) {
        pimc_fields(A, W, Q * sp + c, eff, lab + off[c], itf + c * C, off[c + 1] - off[c]);
    }
    for (int k = 0; k < ncomp; ++k) sv[k] = pimc_gibbs(g, W, eff[k]);
    for (int c = 0; c < Q; ++c) {
        const int *l = lab + off[c];
        if (!pimc_store(W, Q * sp + c, itf + c * C, off[c + 1] - off[c],
                        [&](int d) { return sv[l[d]]; })) {
            W.overflow = true;
            return;
        }
    }
}

template <bool CHAIN>
__global__ void __launch_bounds__(64) pimc_kernel(PimcArgs A) {
    const int R = A.num_samples;
    const int n = A.n;
    const int slot = A.shared_stream ? 0 : (int)(blockIdx.x * blockDim.x + threadIdx.x);
    if (slot >= R) return;
    if (A.shared_stream && (blockIdx.x != 0 || threadIdx.x != 0)) return;
    const int first = slot;
    const int last = A.shared_stream ? R : first + 1;
    const int points = A.interval ? 1 + (A.num_betas - 1) / A.interval : 0;
    const int Q = CHAIN ? A.qpc : 1;
    const int C = A.cap_props + A.cap_breaks;
    int32_t *si = A.scratch_i + (int64_t)slot * A.scratch_ints;
    int32_t *props = si;
    int32_t *itf = props + A.cap_props;
    int32_t *sv = itf + Q * C;
    int32_t *off = sv + Q * C;
    int32_t *lab = off + Q + 1;
    int32_t *parent = lab + Q * C;
    int32_t *pair = parent + Q * C;
    double *eff = A.scratch_d + (int64_t)slot * A.scratch_doubles;
    PimcRng g;
    g.mt = A.mt + (int64_t)slot * kMtWords;
    PimcWorld W;
    W.cap = A.cap_breaks;
    W.near = 0;
    W.overflow = false;
    for (int r = first; r < last && !W.overflow; ++r) {
        if (r == first) g.seed(A.seeds[A.shared_stream ? 0 : r]);  // localPIMC.cpp:578-587
        W.s = A.states + (int64_t)r * n;
        W.cnt = A.counts + (int64_t)r * n;
        W.brk = A.breaks + (int64_t)r * n * A.cap_breaks;
        int8_t *stats = A.stats ? A.stats + (int64_t)r * points * n : nullptr;
        for (int b = 0; b < A.num_betas && !W.overflow; ++b) {
            W.gamma = __ldg(&A.hd[b]);
            W.beta = __ldg(&A.hp[b]);
            const int64_t updates = (int64_t)A.sweeps_per_beta * n;
            for (int64_t k = 0; k < updates && !W.overflow; ++k) {
                if (CHAIN)
                    pimc_chain_update(A, g, W, g.below((uint32_t)A.chains), props, itf, off, lab,
                                      parent, sv, pair, eff);
                else
                    pimc_qubit_update(A, g, W, g.below((uint32_t)n), props, itf, sv, eff);
            }
            if (stats && b % A.interval == 0) {
                for (int v = 0; v < n; ++v) stats[v] = W.s[v];
                stats += n;
            }
        }
        double e = 0.0;  // localPIMC.cpp:59-75
        for (int v = 0; v < n; ++v)
            e = __dadd_rn(e, __dmul_rn((double)W.s[v], __ldg(&A.h[v])));
        for (int64_t c = 0; c < A.m; ++c)
            e = __dadd_rn(e, __dmul_rn(__dmul_rn((double)W.s[__ldg(&A.cu[c])], __ldg(&A.cw[c])),
                                       (double)W.s[__ldg(&A.cv[c])]));
        A.energies[r] = e;
    }
    if (W.overflow) atomicExch(A.overflow, 1);
    if (W.near) atomicAdd(A.near, (unsigned long long)W.near);
}

}  // namespace b200sa
