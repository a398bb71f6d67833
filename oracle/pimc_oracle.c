/* CPU restatement of the reference's path-integral Monte Carlo annealing
 * (dwave-samplers 1.8.0, dwave/samplers/sqa/src/localPIMC.cpp).
 * TEST INFRASTRUCTURE ONLY: the checker for b200sa_path_anneal, never the
 * thing measured or shipped.
 *
 * Followed parts (file:line in localPIMC.cpp unless noted):
 *   general_simulated_annealing :585-715   adjacency in coupler input order,
 *                                           one generator seeded once per call,
 *                                           samples in order, energy per sample
 *   run (schedule loop)           :126-157  Hd drives the loop, Hp = invTemp,
 *                                           sweeps_per_beta * n updates per step
 *   qubitUpdate                   :361-393  single-qubit Swendsen-Wang update
 *   chainUpdate                   :395-464  multi-qubit update over a chain
 *   makeDomainGraph               :474-541
 *   addHToEffectiveField          :277-295, addJToEffectiveField :297-359
 *   makeBreakProposals            :543-555
 *   GibbsSamplePM1 / pNotJoin     :568-576
 *   get_state_energy              :59-75
 *
 * The generator is std::mt19937 from libstdc++ (GCC 13), through two of its
 * distributions; their published algorithms are restated here:
 *   mt19937       Matsumoto & Nishimura (1998), 32-bit, seed by the standard's
 *                 linear recurrence (multiplier 1812433253)
 *   uniform_int_distribution<int>(0, n-1) with a 32-bit generator: Lemire's
 *                 nearly divisionless method (ACM TOMACS 29(1), 2019) on the
 *                 64-bit product of one draw and n
 *   uniform_real_distribution<double>(a, b): generate_canonical<double, 53>
 *                 = (d1 + d2 * 2^32) / 2^64 from two draws (1 - 2^-53 when that
 *                 rounds to 1), then canonical * (b - a) + a
 *
 * Quantum initial states (project_inputs false) read num_breaks[v] break
 * positions for each variable v.  The reference instead reads num_variables
 * positions per variable into a list sized num_breaks[v]
 * (localPIMC.cpp:164-176), which is only well defined when every
 * num_breaks[v] equals num_variables; both agree in that case.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define PIMC_SLICES 65536 /* numTrotterSlices, localPIMC.h:88 */

/* ---- std::mt19937 ---------------------------------------------------- */
typedef struct {
    uint32_t mt[624];
    int idx;
} pimc_mt;

static void mt_seed(pimc_mt *g, uint32_t seed) {
    g->mt[0] = seed;
    for (int i = 1; i < 624; ++i)
        g->mt[i] = 1812433253u * (g->mt[i - 1] ^ (g->mt[i - 1] >> 30)) + (uint32_t)i;
    g->idx = 624;
}

static uint32_t mt_next(pimc_mt *g) {
    if (g->idx >= 624) {
        for (int i = 0; i < 624; ++i) {
            const uint32_t y = (g->mt[i] & 0x80000000u) | (g->mt[(i + 1) % 624] & 0x7fffffffu);
            g->mt[i] = g->mt[(i + 397) % 624] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
        }
        g->idx = 0;
    }
    uint32_t y = g->mt[g->idx++];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
}

/* generate_canonical<double, 53> */
static double mt_canonical(pimc_mt *g) {
    const double lo = (double)mt_next(g);
    const double hi = (double)mt_next(g);
    const double sum = lo + hi * 4294967296.0;
    const double r = sum / 18446744073709551616.0;
    return r >= 1.0 ? 1.0 - 1.1102230246251565e-16 : r; /* nextafter(1, 0) */
}

/* uniform_int_distribution<int>(0, range - 1), range >= 1 */
static int mt_below(pimc_mt *g, uint32_t range) {
    uint64_t prod = (uint64_t)mt_next(g) * range;
    uint32_t low = (uint32_t)prod;
    if (low < range) {
        const uint32_t threshold = (uint32_t)(-range) % range;
        while (low < threshold) {
            prod = (uint64_t)mt_next(g) * range;
            low = (uint32_t)prod;
        }
    }
    return (int)(prod >> 32);
}

/* ---- problem and world lines ------------------------------------------ */
typedef struct {
    int n;
    int *start, *deg, *col; /* adjacency in coupler input order */
    double *w;
    const double *h;
    double jchain;
    int qpc, qpu;
} pimc_problem;

typedef struct {
    int8_t *s;     /* firstSlice */
    int *cnt;      /* breaks per variable */
    int **brk;     /* break positions, increasing */
    int *cap;
    double beta;   /* invTemp */
    double gamma;  /* invTempGamma */
    pimc_mt g;
    int overflow;
} pimc_world;

static void push_break(pimc_world *W, int v, int pos) {
    if (W->cnt[v] == W->cap[v]) {
        W->cap[v] = W->cap[v] ? 2 * W->cap[v] : 8;
        W->brk[v] = (int *)realloc(W->brk[v], sizeof(int) * (size_t)W->cap[v]);
    }
    W->brk[v][W->cnt[v]++] = pos;
}

/* Growable int list for the per-update scratch. */
typedef struct {
    int *a;
    int n, cap;
} ilist;

static void il_push(ilist *l, int x) {
    if (l->n == l->cap) {
        l->cap = l->cap ? 2 * l->cap : 16;
        l->a = (int *)realloc(l->a, sizeof(int) * (size_t)l->cap);
    }
    l->a[l->n++] = x;
}

/* std::merge: on equal values the element of the first range comes first. */
static void merge_into(ilist *out, const int *a, int na, const int *b, int nb) {
    int i = 0, j = 0;
    out->n = 0;
    while (i < na && j < nb) {
        if (b[j] < a[i])
            il_push(out, b[j++]);
        else
            il_push(out, a[i++]);
    }
    while (i < na) il_push(out, a[i++]);
    while (j < nb) il_push(out, b[j++]);
}

/* makeBreakProposals: exponential gaps of scale slices / gamma. */
static void make_proposals(pimc_world *W, ilist *out) {
    const double scale = (double)PIMC_SLICES / W->gamma;
    out->n = 0;
    double position = -scale * log(mt_canonical(&W->g));
    while (position < (double)PIMC_SLICES) {
        il_push(out, (int)position);
        position = -scale * log(mt_canonical(&W->g)) + (double)out->a[out->n - 1] + 1.0;
    }
}

/* Interfaces of one qubit: proposals merged with its breaks, or the single
 * book-keeping value when there is at most one of them together. */
static void interfaces(pimc_world *W, int q, ilist *props, ilist *itf) {
    make_proposals(W, props);
    if (props->n + W->cnt[q] > 1) {
        merge_into(itf, props->a, props->n, W->brk[q], W->cnt[q]);
    } else {
        itf->n = 0;
        il_push(itf, PIMC_SLICES);
    }
}

/* addHToEffectiveField; lab maps a domain to its accumulator (NULL: itself). */
static void add_h(double *eff, const int *lab, const int *itf, int nd, double H) {
    H /= (double)PIMC_SLICES;
    const int d0 = lab ? lab[0] : 0;
    eff[d0] += (double)(PIMC_SLICES + itf[0] - itf[nd - 1]) * H;
    for (int i = 1; i < nd; ++i) eff[lab ? lab[i] : i] += (double)(itf[i] - itf[i - 1]) * H;
}

/* addJToEffectiveField: the neighbour's spin, flipped at each of its breaks,
 * over the domains of this qubit. */
static void add_j(double *eff, const int *lab, const int *itf, int nd, const int *nb, int nnb,
                  double Js, ilist *pair) {
    Js /= (double)PIMC_SLICES;
    merge_into(pair, nb, nnb, itf, nd);
    const int *p = pair->a;
    const int L = pair->n;
    const int d0 = lab ? lab[0] : 0;
    eff[d0] += (double)(PIMC_SLICES + p[0] - p[L - 1]) * Js;
    int i = 0, oi = 0;
    for (; i + 1 < L; ++i) {
        if (p[i] == itf[oi]) {
            if (++oi == nd) break;
        } else {
            Js *= -1;
        }
        eff[lab ? lab[oi] : oi] += (double)(p[i + 1] - p[i]) * Js;
    }
    for (; i + 1 < L; ++i) {
        eff[d0] += (double)(p[i + 1] - p[i]) * Js;
        Js *= -1;
    }
}

static int gibbs_pm1(pimc_world *W, double field) {
    const double thr = mt_canonical(&W->g) * 2.0 + -1.0; /* uniform(-1, 1) */
    return tanh(W->beta * field) > thr ? -1 : 1;
}

static double p_not_join(const pimc_problem *P, const pimc_world *W, int overlaps) {
    return exp((2.0 * P->jchain * (double)overlaps * W->beta) / (double)PIMC_SLICES);
}

typedef struct {
    ilist props, pair;
    ilist *itf;    /* per chain qubit */
    double *eff;
    int eff_cap;
    int *lab, *parent, *sv, lab_cap;
} pimc_scratch;

static void ensure_eff(pimc_scratch *S, int n) {
    if (n > S->eff_cap) {
        S->eff_cap = 2 * n;
        S->eff = (double *)realloc(S->eff, sizeof(double) * (size_t)S->eff_cap);
    }
}

static void ensure_lab(pimc_scratch *S, int n) {
    if (n > S->lab_cap) {
        S->lab_cap = 2 * n;
        S->lab = (int *)realloc(S->lab, sizeof(int) * (size_t)S->lab_cap);
        S->parent = (int *)realloc(S->parent, sizeof(int) * (size_t)S->lab_cap);
        S->sv = (int *)realloc(S->sv, sizeof(int) * (size_t)S->lab_cap);
    }
}

/* qubitUpdate (localPIMC.cpp:361-393). */
static void qubit_update(const pimc_problem *P, pimc_world *W, pimc_scratch *S, int sp) {
    ilist *itf = &S->itf[0];
    interfaces(W, sp, &S->props, itf);
    const int nd = itf->n;
    ensure_eff(S, nd);
    for (int i = 0; i < nd; ++i) S->eff[i] = 0.0;
    add_h(S->eff, NULL, itf->a, nd, P->h[sp]);
    for (int k = 0; k < P->deg[sp]; ++k) {
        const int nb = P->col[P->start[sp] + k];
        add_j(S->eff, NULL, itf->a, nd, W->brk[nb], W->cnt[nb],
              (double)W->s[nb] * P->w[P->start[sp] + k], &S->pair);
    }
    int sv = gibbs_pm1(W, S->eff[0]);
    const int first = sv;
    W->s[sp] = (int8_t)sv;
    W->cnt[sp] = 0;
    for (int i = 1; i < nd; ++i) {
        if (sv * gibbs_pm1(W, S->eff[i]) != 1) {
            sv = -sv;
            push_break(W, sp, itf->a[i - 1]);
        }
    }
    if (sv != first) push_break(W, sp, itf->a[nd - 1]);
}

static int uf_find(int *parent, int x) {
    while (parent[x] != x) {
        parent[x] = parent[parent[x]];
        x = parent[x];
    }
    return x;
}

static void uf_join(int *parent, int a, int b) {
    a = uf_find(parent, a);
    b = uf_find(parent, b);
    if (a != b) parent[a < b ? b : a] = a < b ? a : b;
}

/* makeDomainGraph (localPIMC.cpp:474-541) for chain qubits c and c + 1;
 * joins go straight into the union-find forest. */
static void domain_graph(const pimc_problem *P, pimc_world *W, pimc_scratch *S, int z, int f,
                         int sp, int c) {
    const int q = sp * P->qpc + c;
    int s0s1 = (int)W->s[q] * (int)W->s[q + 1];
    const ilist *A = &S->itf[c], *B = &S->itf[c + 1];
    merge_into(&S->pair, A->a, A->n, B->a, B->n);
    const int *p = S->pair.a;
    int L = S->pair.n;
    if (p[0] == PIMC_SLICES) {
        if (s0s1 == 1 && p_not_join(P, W, PIMC_SLICES) < mt_canonical(&W->g))
            uf_join(S->parent, z, f);
        return;
    }
    if (p[L - 1] == PIMC_SLICES) --L;
    if (s0s1 == 1 && p_not_join(P, W, PIMC_SLICES - p[L - 1] + p[0]) < mt_canonical(&W->g))
        uf_join(S->parent, z, f);
    int p0 = 0, e0 = 0, p1 = 0, e1 = 0;
    int valid0 = A->a[0] != PIMC_SLICES;
    int i = 0;
    while (++i < L) {
        if (valid0 && p[i - 1] == A->a[p0]) {
            if (A->n == ++p0) {
                valid0 = 0;
                p0 = 0;
            }
            if (W->cnt[q] > e0 && p[i - 1] == W->brk[q][e0]) {
                s0s1 = -s0s1;
                e0++;
            }
        } else {
            if (B->n == ++p1) p1 = 0;
            if (W->cnt[q + 1] > e1 && p[i - 1] == W->brk[q + 1][e1]) {
                s0s1 = -s0s1;
                e1++;
            }
        }
        if (s0s1 == 1 && p_not_join(P, W, p[i] - p[i - 1]) < mt_canonical(&W->g))
            uf_join(S->parent, z + p0, f + p1);
    }
}

/* chainUpdate (localPIMC.cpp:395-464).  Components are numbered in order of
 * their smallest domain, as the reference's depth-first labelling from roots
 * 0, 1, ... does. */
static void chain_update(const pimc_problem *P, pimc_world *W, pimc_scratch *S, int sp) {
    const int Q = P->qpc;
    int total = 0;
    int *off = (int *)malloc(sizeof(int) * (size_t)Q);
    for (int c = 0; c < Q; ++c) {
        interfaces(W, Q * sp + c, &S->props, &S->itf[c]);
        off[c] = total;
        total += S->itf[c].n;
    }
    ensure_lab(S, total);
    for (int d = 0; d < total; ++d) S->parent[d] = d;
    for (int c = 0; c + 1 < Q; ++c) domain_graph(P, W, S, off[c], off[c + 1], sp, c);
    int ncomp = 0;
    for (int d = 0; d < total; ++d) S->sv[d] = -1; /* label of each root */
    for (int d = 0; d < total; ++d) {
        const int r = uf_find(S->parent, d);
        if (S->sv[r] < 0) S->sv[r] = ncomp++;
        S->lab[d] = S->sv[r];
    }
    ensure_eff(S, ncomp);
    for (int k = 0; k < ncomp; ++k) S->eff[k] = 0.0;
    for (int c = 0; c < Q; ++c) {
        const int q = Q * sp + c;
        const ilist *itf = &S->itf[c];
        add_h(S->eff, S->lab + off[c], itf->a, itf->n, P->h[q]);
        for (int k = 0; k < P->deg[q]; ++k) {
            const int nb = P->col[P->start[q] + k];
            add_j(S->eff, S->lab + off[c], itf->a, itf->n, W->brk[nb], W->cnt[nb],
                  (double)W->s[nb] * P->w[P->start[q] + k], &S->pair);
        }
    }
    for (int k = 0; k < ncomp; ++k) S->sv[k] = gibbs_pm1(W, S->eff[k]);
    for (int c = 0; c < Q; ++c) {
        const int q = Q * sp + c;
        const ilist *itf = &S->itf[c];
        const int *lab = S->lab + off[c];
        W->s[q] = (int8_t)S->sv[lab[0]];
        W->cnt[q] = 0;
        int sv = W->s[q];
        for (int d = 1; d < itf->n; ++d) {
            if (sv * S->sv[lab[d]] != 1) {
                sv = -sv;
                push_break(W, q, itf->a[d - 1]);
            }
        }
        if (sv != W->s[q]) push_break(W, q, itf->a[itf->n - 1]);
    }
    free(off);
}

static double pimc_energy(int n, const int8_t *s, const double *h, long m, const int *u,
                          const int *v, const double *J) {
    double e = 0.0;
    for (int i = 0; i < n; ++i) e += s[i] * h[i];
    for (long c = 0; c < m; ++c) e += s[u[c]] * J[c] * s[v[c]];
    return e;
}

/* One reference call: samples annealed in order from one generator.
 *   states      [R*n] int8, in/out
 *   num_breaks  [R*n] in (project_inputs == 0) and out (project_outputs == 0)
 *   breaks_in   flat positions, num_breaks[r][v] per variable in order
 *   breaks_out  [R*n*max_out]: sample r, variable v at ((r*n)+v)*max_out
 *   statistics  [R*points*n] or NULL
 * Returns R, or -1 on bad input, -2 when a variable ends with more than
 * max_out breaks (breaks_out too small). */
int pimc_oracle_run(int n, const double *h, long m, const int *u, const int *v, const double *J,
                    int R, int8_t *states, double *energies, int spb, int nbetas,
                    const double *hp, const double *hd, double jchain, int qpc, int qpu,
                    uint32_t seed, int project_inputs, int project_outputs, int *num_breaks,
                    const int *breaks_in, int *breaks_out, int max_out, int8_t *statistics,
                    int interval) {
    if (qpc < 1) return -1;
    for (long c = 0; c < m; ++c)
        if (u[c] < 0 || v[c] < 0 || u[c] >= n || v[c] >= n) return -1;
    pimc_problem P;
    memset(&P, 0, sizeof P);
    P.n = n;
    P.h = h;
    P.jchain = jchain;
    P.qpc = qpc;
    P.qpu = qpu;
    P.deg = (int *)calloc((size_t)n + 1, sizeof(int));
    P.start = (int *)calloc((size_t)n + 1, sizeof(int));
    P.col = (int *)malloc(sizeof(int) * (size_t)(2 * m + 1));
    P.w = (double *)malloc(sizeof(double) * (size_t)(2 * m + 1));
    for (long c = 0; c < m; ++c) {
        P.deg[u[c]]++;
        P.deg[v[c]]++;
    }
    for (int i = 0; i < n; ++i) P.start[i + 1] = P.start[i] + P.deg[i];
    int *fill = (int *)calloc((size_t)n + 1, sizeof(int));
    for (long c = 0; c < m; ++c) { /* neighbors[u].push(v); neighbors[v].push(u) */
        P.col[P.start[u[c]] + fill[u[c]]] = v[c];
        P.w[P.start[u[c]] + fill[u[c]]++] = J[c];
        P.col[P.start[v[c]] + fill[v[c]]] = u[c];
        P.w[P.start[v[c]] + fill[v[c]]++] = J[c];
    }
    free(fill);
    pimc_world W;
    memset(&W, 0, sizeof W);
    W.s = (int8_t *)calloc((size_t)n + 1, 1);
    W.cnt = (int *)calloc((size_t)n + 1, sizeof(int));
    W.cap = (int *)calloc((size_t)n + 1, sizeof(int));
    W.brk = (int **)calloc((size_t)n + 1, sizeof(int *));
    mt_seed(&W.g, seed);
    pimc_scratch S;
    memset(&S, 0, sizeof S);
    S.itf = (ilist *)calloc((size_t)qpc, sizeof(ilist));
    const int points = interval ? 1 + (nbetas - 1) / interval : 0;
    const int chains = n / qpc;
    long in_pos = 0;
    int rc = R;
    for (int r = 0; r < R; ++r) {
        int8_t *st = states + (size_t)r * n;
        for (int i = 0; i < n; ++i) {
            W.s[i] = st[i];
            W.cnt[i] = 0;
            if (!project_inputs)
                for (int k = 0; k < num_breaks[(size_t)r * n + i]; ++k)
                    push_break(&W, i, breaks_in[in_pos++]);
        }
        int8_t *stats = statistics ? statistics + (size_t)r * points * n : NULL;
        for (int b = 0; b < nbetas; ++b) {
            W.gamma = hd[b];
            W.beta = hp[b];
            const long updates = (long)spb * n;
            for (long k = 0; k < updates; ++k) {
                if (qpu == 1)
                    qubit_update(&P, &W, &S, mt_below(&W.g, (uint32_t)n));
                else
                    chain_update(&P, &W, &S, mt_below(&W.g, (uint32_t)chains));
            }
            if (stats && b % interval == 0) {
                memcpy(stats, W.s, (size_t)n);
                stats += n;
            }
        }
        memcpy(st, W.s, (size_t)n);
        energies[r] = pimc_energy(n, st, h, m, u, v, J);
        if (!project_outputs) {
            for (int i = 0; i < n; ++i) {
                num_breaks[(size_t)r * n + i] = W.cnt[i];
                if (W.cnt[i] > max_out) {
                    rc = -2;
                    continue;
                }
                memcpy(breaks_out + ((size_t)r * n + i) * (size_t)max_out, W.brk[i],
                       sizeof(int) * (size_t)W.cnt[i]);
            }
        }
    }
    for (int i = 0; i < n; ++i) free(W.brk[i]);
    free(W.brk);
    free(W.cnt);
    free(W.cap);
    free(W.s);
    for (int c = 0; c < qpc; ++c) free(S.itf[c].a);
    free(S.itf);
    free(S.props.a);
    free(S.pair.a);
    free(S.eff);
    free(S.lab);
    free(S.parent);
    free(S.sv);
    free(P.deg);
    free(P.start);
    free(P.col);
    free(P.w);
    return rc;
}

/* First `count` outputs of std::mt19937(seed), for pinning the generator. */
void pimc_oracle_mt(uint32_t seed, int count, uint32_t *out) {
    pimc_mt g;
    mt_seed(&g, seed);
    for (int i = 0; i < count; ++i) out[i] = mt_next(&g);
}
