// Host-side packing: argument validation, order-preserving adjacency,
// per-variable speculation info and the RNG jump matrix.
#include "pack.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstdio>

#include "sa_types.h"

namespace b200sa {

int validate_problem(const b200sa_problem &p, std::string &msg) {
    char buf[256];
    if (p.num_vars < 0 || p.num_couplers < 0 || p.num_reads < 0) {
        msg = "negative size";
        return B200SA_EINVAL;
    }
    if (p.num_couplers > (int64_t)INT32_MAX / 2) {
        msg = "too many couplers";
        return B200SA_EINVAL;
    }
    if (p.num_vars > 0 && !p.h) {
        msg = "h is NULL";
        return B200SA_EINVAL;
    }
    if (p.num_couplers > 0 &&
        (!p.coupler_starts || !p.coupler_ends || !p.coupler_weights)) {
        msg = "coupler arrays are NULL";
        return B200SA_EINVAL;
    }
    if (p.sweeps_per_beta < 0 || p.num_betas < 0 ||
        (p.num_betas > 0 && !p.beta_schedule)) {
        msg = "bad beta schedule";
        return B200SA_EINVAL;
    }
    if (p.varorder != B200SA_SEQUENTIAL && p.varorder != B200SA_RANDOM) {
        msg = "varorder must be 0 (sequential) or 1 (random)";
        return B200SA_EINVAL;
    }
    if (p.proposal != B200SA_GIBBS && p.proposal != B200SA_METROPOLIS) {
        msg = "proposal must be 0 (Gibbs) or 1 (Metropolis)";
        return B200SA_EINVAL;
    }
    // cpu_sa.cpp:302-304 (the reference throws; here it is an error code).
    std::vector<uint32_t> deg((size_t)std::max(p.num_vars, 0), 0);
    for (int64_t c = 0; c < p.num_couplers; ++c) {
        const int32_t a = p.coupler_starts[c], b = p.coupler_ends[c];
        if (a < 0 || b < 0 || a >= p.num_vars || b >= p.num_vars) {
            std::snprintf(buf, sizeof(buf),
                          "coupler indexes contain an invalid variable "
                          "(coupler %lld: %d, %d; num_vars %d)",
                          (long long)c, a, b, p.num_vars);
            msg = buf;
            return B200SA_EINVAL;
        }
        if (++deg[a] > kMaxDegree || ++deg[b] > kMaxDegree) {
            msg = "a variable has more than 2^24-1 adjacency entries";
            return B200SA_EINVAL;
        }
    }
    return B200SA_OK;
}

void pack_adjacency(const b200sa_problem &p, PackedAdjacency &out) {
    const int32_t n = p.num_vars;
    const int64_t m = p.num_couplers;
    out.row.assign((size_t)n + 1, 0);
    out.col.resize((size_t)(2 * m));
    out.w.resize((size_t)(2 * m));
    out.vinfo.assign((size_t)n * 2, 0);
    for (int64_t c = 0; c < m; ++c) {
        out.row[(size_t)p.coupler_starts[c] + 1]++;
        out.row[(size_t)p.coupler_ends[c] + 1]++;
    }
    for (int32_t i = 0; i < n; ++i) out.row[i + 1] += out.row[i];
    // Counting-sort fill in coupler order: the same per-variable order as the
    // reference's push_back loop (cpu_sa.cpp:298-316).
    std::vector<int32_t> cur(out.row.begin(), out.row.end() - 1);
    for (int64_t c = 0; c < m; ++c) {
        const int32_t a = p.coupler_starts[c], b = p.coupler_ends[c];
        const double J = p.coupler_weights[c];
        int32_t k = cur[a]++;
        out.col[k] = b;
        out.w[k] = J;
        k = cur[b]++;
        out.col[k] = a;
        out.w[k] = J;
    }
    // Speculation record: nearest later neighbour; repeated targets; pairs
    // of variables less than 32 apart with a common neighbour.
    out.share.assign((size_t)n, 0u);
    out.dist.assign((size_t)n, 0u);
    {
        std::vector<int32_t> nb;
        for (int32_t u = 0; u < n; ++u) {
            nb.assign(out.col.begin() + out.row[u], out.col.begin() + out.row[u + 1]);
            std::sort(nb.begin(), nb.end());
            nb.erase(std::unique(nb.begin(), nb.end()), nb.end());
            for (size_t i = 0; i < nb.size(); ++i)
                for (size_t j = i + 1; j < nb.size() && nb[j] - nb[i] < 32; ++j)
                    out.share[nb[i]] |= 1u << (nb[j] - nb[i]);
        }
    }
    std::vector<int32_t> mark((size_t)n, -1);
    int32_t maxdeg = 0;
    bool any_dup = false;
    for (int32_t v = 0; v < n; ++v) {
        uint32_t dist = kDistCap;
        const int32_t e0 = out.row[v], e1 = out.row[v + 1];
        maxdeg = std::max(maxdeg, e1 - e0);
        for (int32_t e = e0; e < e1; ++e) {
            const int32_t u = out.col[e];
            if (u > v) dist = std::min<uint32_t>(dist, (uint32_t)(u - v));
            if (mark[u] == v) {
                any_dup = true;
                out.share[v] |= 1u;
            }
            mark[u] = v;
        }
        out.vinfo[2 * (size_t)v] = (uint32_t)e0;
        out.vinfo[2 * (size_t)v + 1] = (uint32_t)(e1 - e0);
        out.dist[v] = (uint8_t)dist;
    }
    out.max_degree = maxdeg;
    out.any_dup = any_dup;
    // Back-neighbour records.  Resolution pays when later lanes of a window
    // often depend on earlier ones: on average at least one back neighbour in
    // two variables (measured on random-regular batches: one in four resolved
    // problems that ran 1-2% faster without), and no list naming a target
    // twice (the in-register corrections add one term per neighbour).
    out.back.assign((size_t)n * 2, 0u);
    out.bw.clear();
    out.bw_src.clear();
    for (int32_t v = 0; v < n; ++v) {
        uint32_t mask = 0;
        int32_t at[32];
        for (int32_t e = out.row[v]; e < out.row[v + 1]; ++e) {
            const int32_t o = v - out.col[e];
            if (o > 0 && o < 32) {
                mask |= 1u << o;
                at[o] = e;
            }
        }
        out.back[2 * (size_t)v] = mask;
        out.back[2 * (size_t)v + 1] = (uint32_t)out.bw.size();
        for (int o = 31; o >= 1; --o) {
            if (!((mask >> o) & 1u)) continue;
            out.bw.push_back(out.w[(size_t)at[o]]);
            out.bw_src.push_back(at[o]);
        }
    }
    out.resolve = !any_dup && n > 0 && 2 * out.bw.size() >= (size_t)n;
    {
        std::vector<int32_t> offs(out.col.size());
        for (int32_t v = 0; v < n; ++v)
            for (int32_t e = out.row[v]; e < out.row[v + 1]; ++e)
                offs[(size_t)e] = std::abs(out.col[e] - v);
        int32_t b = 32;
        if (!offs.empty()) {
            const size_t k = std::min(offs.size() - 1, (offs.size() * 97) / 100);
            std::nth_element(offs.begin(), offs.begin() + (std::ptrdiff_t)k, offs.end());
            b = std::max<int32_t>(32, offs[k]);
        }
        int64_t w = 1;
        while (w < 2 * (int64_t)b + 128) w <<= 1;
        out.band_b = b;
        out.band_w = (w <= kBandMaxSlots && 2 * w <= (int64_t)n) ? (int32_t)w : 0;
    }
    out.dense = out.resolve && n <= kDenseMaxN && 16 * (size_t)m >= (size_t)n * (size_t)n;
    out.dense_w.clear();
    out.dense_bits.clear();
    if (out.dense) {
        out.dense_w.assign((size_t)n * (size_t)n, 0.0);
        out.dense_bits.assign((size_t)n * 4, 0u);
        for (int32_t j = 0; j < n; ++j)
            for (int32_t e = out.row[j]; e < out.row[j + 1]; ++e) {
                const int32_t x = out.col[e];
                out.dense_w[(size_t)j * n + x] = out.w[e];
                out.dense_bits[(size_t)j * 4 + (x >> 5)] |= 1u << (x & 31);
            }
    }
    out.regular_degree = 0;
    if (n > 0 && maxdeg > 0 && maxdeg <= 32) {
        bool reg = true;
        for (int32_t v = 0; v < n && reg; ++v) reg = (out.row[v + 1] - out.row[v]) == maxdeg;
        if (reg) out.regular_degree = maxdeg;
    }
}

// One xorshift128+ state transition (cpu_sa.cpp:27-34 without the output).
static inline void xs_advance(uint64_t &s0, uint64_t &s1) {
    uint64_t a = s0;
    const uint64_t b = s1;
    s0 = b;
    a ^= a << 23;
    s1 = a ^ b ^ (a >> 17) ^ (b >> 26);
}

void rng_jump_columns(int64_t steps, uint32_t out[128][4]) {
    for (int bit = 0; bit < 128; ++bit) {
        uint64_t s0 = bit < 64 ? (1ull << bit) : 0;
        uint64_t s1 = bit < 64 ? 0 : (1ull << (bit - 64));
        for (int64_t k = 0; k < steps; ++k) xs_advance(s0, s1);
        out[bit][0] = (uint32_t)s0;
        out[bit][1] = (uint32_t)(s0 >> 32);
        out[bit][2] = (uint32_t)s1;
        out[bit][3] = (uint32_t)(s1 >> 32);
    }
}

void rng_jump_nibbles(const uint32_t cols[128][4], uint32_t out[][4]) {
    for (int k = 0; k < kJumpNibbles; ++k) {
        for (int v = 0; v < 16; ++v) {
            uint32_t acc[4] = {0, 0, 0, 0};
            for (int b = 0; b < 4; ++b) {
                if (!((v >> b) & 1)) continue;
                for (int w = 0; w < 4; ++w) acc[w] ^= cols[4 * k + b][w];
            }
            for (int w = 0; w < 4; ++w) out[k * 16 + v][w] = acc[w];
        }
    }
}

}  // namespace b200sa
