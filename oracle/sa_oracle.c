/*
 * CPU restatement of the reference simulated-annealing sweep.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity oracle for the CUDA
 * sampler: only tests, the smoke check and the CPU-baseline leg of the
 * benchmark load it.  The product library never links or calls it.
 *
 * It restates, in plain C, the algorithm of dwave-samplers 1.8.0
 * (dwave/samplers/sa/src/cpu_sa.cpp); every function names the lines it
 * follows.  It is pinned against the reference extension built from source
 * (oracle/build_ref.sh) by tests/test_oracle.py and against the committed
 * golden vectors in tests/golden/.
 *
 * Two seeding modes:
 *   num_seeds == 1         : one xorshift128+ stream seeded once per call and
 *                            continued across reads (cpu_sa.cpp:283-284, 321-358)
 *   num_seeds == num_reads : read r is an independent call with num_samples=1
 *                            and seed=seeds[r] (the per-read contract).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORACLE_EINVAL (-1)
#define ORACLE_ENOMEM (-2)

/* xorshift128+ step, cpu_sa.cpp:27-34.  Returns s1_new + s1_old. */
static inline uint64_t rng_next(uint64_t st[2]) {
    uint64_t a = st[0];
    const uint64_t b = st[1];
    st[0] = b;
    a ^= a << 23;
    st[1] = a ^ b ^ (a >> 17) ^ (b >> 26);
    return st[1] + b;
}

/* Seeding, cpu_sa.cpp:283-284: zero is replaced by 2^64-1. */
static inline void rng_seed(uint64_t st[2], uint64_t seed) {
    st[0] = seed ? seed : UINT64_MAX;
    st[1] = 0;
}

/* The reference's RANDMAX ((uint64_t)-1) used as a double operand rounds to
 * 2^64 (cpu_sa.cpp:36, 154, 163). */
static const double RANDMAX_D = 18446744073709551616.0;

typedef struct {
    int n;
    int *row;     /* n+1 offsets */
    int *col;     /* neighbour index, per adjacency entry */
    double *w;    /* coupling, per adjacency entry */
} adjacency;

/* Adjacency in coupler input order, cpu_sa.cpp:298-316: coupler c appends v
 * to u's list and u to v's list (a self-loop appends v twice to its own list).
 * A counting sort over the coupler list reproduces the push_back order. */
static int build_adjacency(adjacency *a, int n, long m, const int *u,
                           const int *v, const double *J) {
    a->n = n;
    a->row = (int *)calloc((size_t)n + 1, sizeof(int));
    a->col = (int *)malloc(sizeof(int) * (size_t)(2 * m + 1));
    a->w = (double *)malloc(sizeof(double) * (size_t)(2 * m + 1));
    int *cur = (int *)malloc(sizeof(int) * ((size_t)n + 1));
    if (!a->row || !a->col || !a->w || !cur) {
        free(cur);
        return ORACLE_ENOMEM;
    }
    for (long c = 0; c < m; c++) {
        if (u[c] < 0 || v[c] < 0 || u[c] >= n || v[c] >= n) {
            free(cur);
            return ORACLE_EINVAL; /* cpu_sa.cpp:302-304 throws here */
        }
        a->row[u[c] + 1]++;
        a->row[v[c] + 1]++;
    }
    for (int i = 0; i < n; i++) a->row[i + 1] += a->row[i];
    memcpy(cur, a->row, sizeof(int) * (size_t)n);
    for (long c = 0; c < m; c++) {
        int k = cur[u[c]]++;
        a->col[k] = v[c];
        a->w[k] = J[c];
        k = cur[v[c]]++;
        a->col[k] = u[c];
        a->w[k] = J[c];
    }
    free(cur);
    return 0;
}

static void free_adjacency(adjacency *a) {
    free(a->row);
    free(a->col);
    free(a->w);
}

/* Energy change of flipping `var`, cpu_sa.cpp:54-74: the local field is
 * summed left to right in adjacency order, then scaled by -2*s. */
static double flip_energy(int var, const int8_t *s, const double *h,
                          const adjacency *a) {
    double f = h[var];
    for (int k = a->row[var]; k < a->row[var + 1]; k++)
        f += s[a->col[k]] * a->w[k];
    return (-2 * s[var]) * f;
}

/* One read, cpu_sa.cpp:93-197.  `order` 0 = sequential, 1 = random;
 * `gibbs` 0 = Metropolis, 1 = Gibbs. */
static void anneal_one(int8_t *s, const double *h, const adjacency *a,
                       int sweeps_per_beta, int num_betas, const double *betas,
                       int order, int gibbs, uint64_t st[2], double *de) {
    const int n = a->n;
    for (int i = 0; i < n; i++) de[i] = flip_energy(i, s, h, a);

    for (int b = 0; b < num_betas; b++) {
        const double beta = betas[b];
        for (int sw = 0; sw < sweeps_per_beta; sw++) {
            const double threshold = 44.36142 / beta; /* cpu_sa.cpp:131 */
            for (int i = 0; i < n; i++) {
                int var = i;
                if (order) var = (int)(rng_next(st) % (uint64_t)n); /* :134-136 */
                if (de[var] >= threshold) continue;                 /* :140 */
                int flip = 0;
                if (!gibbs) { /* Metropolis, :144-158 */
                    if (de[var] <= 0.0) {
                        flip = 1;
                    } else {
                        uint64_t r = rng_next(st);
                        if (exp(-de[var] * beta) * RANDMAX_D > (double)r) flip = 1;
                    }
                } else { /* Gibbs, :159-166 */
                    uint64_t r = rng_next(st);
                    if (RANDMAX_D > (double)r * (1 + exp(de[var] * beta))) flip = 1;
                }
                if (flip) { /* :168-191 */
                    const int8_t mult = (int8_t)(4 * s[var]);
                    for (int k = a->row[var]; k < a->row[var + 1]; k++) {
                        const int nb = a->col[k];
                        de[nb] += mult * a->w[k] * s[nb];
                    }
                    s[var] = (int8_t)(-s[var]);
                    de[var] = -de[var];
                }
            }
        }
    }
}

/* State energy, cpu_sa.cpp:210-227: fields in variable order, then couplers
 * in input order, one running double. */
double sa_oracle_energy(int n, const double *h, long m, const int *u,
                        const int *v, const double *J, const int8_t *s) {
    double e = 0.0;
    for (int i = 0; i < n; i++) e += s[i] * h[i];
    for (long c = 0; c < m; c++) e += s[u[c]] * J[c] * s[v[c]];
    return e;
}

/* Driver, cpu_sa.cpp:253-362.  Returns reads completed (no interrupt here:
 * interrupt polling is host logic tested elsewhere) or a negative error. */
int sa_oracle_run(int n, const double *h, long m, const int *u, const int *v,
                  const double *J, int num_reads, int8_t *states,
                  double *energies, int sweeps_per_beta, int num_betas,
                  const double *betas, const uint64_t *seeds, int num_seeds,
                  int order, int gibbs) {
    if (num_reads < 0 || n < 0 || m < 0) return ORACLE_EINVAL;
    if (num_seeds != 1 && num_seeds != num_reads) return ORACLE_EINVAL;
    if (num_reads == 0 || n == 0) return num_reads;
    adjacency a;
    memset(&a, 0, sizeof(a));
    int rc = build_adjacency(&a, n, m, u, v, J);
    double *de = (double *)malloc(sizeof(double) * (size_t)n);
    if (rc != 0 || !de) {
        free_adjacency(&a);
        free(de);
        return rc ? rc : ORACLE_ENOMEM;
    }
    uint64_t st[2] = {0, 0};
    if (num_seeds == 1) rng_seed(st, seeds[0]);
    for (int r = 0; r < num_reads; r++) {
        if (num_seeds != 1) rng_seed(st, seeds[r]);
        int8_t *s = states + (size_t)r * (size_t)n;
        anneal_one(s, h, &a, sweeps_per_beta, num_betas, betas, order, gibbs,
                   st, de);
        energies[r] = sa_oracle_energy(n, h, m, u, v, J, s);
    }
    free(de);
    free_adjacency(&a);
    return num_reads;
}

/* First `count` xorshift128+ outputs for `seed` (used by RNG unit tests). */
void sa_oracle_rng_stream(uint64_t seed, int count, uint64_t *out) {
    uint64_t st[2];
    rng_seed(st, seed);
    for (int i = 0; i < count; i++) out[i] = rng_next(st);
}

/* ---- Steepest descent: dwave/samplers/greedy/src/descent.cpp ---------------
 * The flip energy (descent.cpp:41-60) and the state energy (:75-93) are the
 * same expressions as cpu_sa.cpp:54-74 and :210-227 above. */

/* Linear-search solver, descent.cpp:117-187: flip the variable with the most
 * negative flip energy (the first such index), update its neighbours with the
 * NEW spin, until no flip energy is negative. */
static unsigned sd_linear(int8_t *s, const double *h, const adjacency *a, double *fe) {
    const int n = a->n;
    if (n < 1) return 0;
    for (int i = 0; i < n; i++) fe[i] = flip_energy(i, s, h, a);
    unsigned steps = 0;
    for (;;) {
        int best = -1;
        double best_e = 0;
        for (int i = 0; i < n; i++)
            if (fe[i] < best_e) {
                best_e = fe[i];
                best = i;
            }
        if (best < 0) break;
        s[best] = (int8_t)(s[best] * -1);                        /* :168 */
        fe[best] *= -1;                                          /* :172 */
        for (int k = a->row[best]; k < a->row[best + 1]; k++) { /* :174-182 */
            const int nb = a->col[k];
            fe[nb] -= 4 * s[best] * a->w[k] * s[nb];
        }
        steps++;
    }
    return steps;
}

/* Ordered-set solver, descent.cpp:210-289: the same selection (least flip
 * energy, ties to the lower index), neighbours updated with the OLD spin
 * before the flip, and the flipped variable's entry then set to the negated
 * value it had before the neighbour loop. */
static unsigned sd_sparse(int8_t *s, const double *h, const adjacency *a, double *fe) {
    const int n = a->n;
    if (n < 1) return 0;
    for (int i = 0; i < n; i++) fe[i] = flip_energy(i, s, h, a);
    unsigned steps = 0;
    for (;;) {
        int best = 0;
        double best_e = fe[0];
        for (int i = 1; i < n; i++)
            if (fe[i] < best_e) {
                best_e = fe[i];
                best = i;
            }
        if (best_e >= 0) break;                                  /* :244 */
        for (int k = a->row[best]; k < a->row[best + 1]; k++) { /* :255-277 */
            const int nb = a->col[k];
            fe[nb] = fe[nb] + 4 * s[best] * a->w[k] * s[nb];
        }
        s[best] = (int8_t)(s[best] * -1);                        /* :280 */
        fe[best] = best_e * -1;                                  /* :283-285 */
        steps++;
    }
    return steps;
}

/* Driver, descent.cpp:315-405: each sample descends from its row of
 * `states` (overwritten), then its energy; steps per sample. */
int sd_oracle_run(int n, const double *h, long m, const int *u, const int *v,
                  const double *J, int num_samples, int8_t *states, double *energies,
                  unsigned *steps, int large_sparse_opt) {
    adjacency a;
    int rc = build_adjacency(&a, n, m, u, v, J);
    if (rc) {
        free_adjacency(&a);
        return rc;
    }
    double *fe = (double *)malloc(sizeof(double) * ((size_t)n + 1));
    if (!fe) {
        free_adjacency(&a);
        return ORACLE_ENOMEM;
    }
    for (int r = 0; r < num_samples; r++) {
        int8_t *s = states + (size_t)r * (size_t)n;
        steps[r] = large_sparse_opt ? sd_sparse(s, h, &a, fe) : sd_linear(s, h, &a, fe);
        energies[r] = sa_oracle_energy(n, h, m, u, v, J, s);
    }
    free(fe);
    free_adjacency(&a);
    return num_samples;
}

/* ---- Rotor-model annealing (SQA): dwave/samplers/sqa/src/cpu_rotormc.cpp ----
 * States are uint8 angles theta = 2*pi*index/256, with cos and |sin| tables
 * computed as at cpu_rotormc.cpp:377-383.  Proposals (cpu_rotormc.h enum):
 * 0 GibbsNonErgodic, 1 MetropolisNonErgodic, 2 MetropolisUniform,
 * 3 MetropolisTF. */

static const double RMC_PI = 3.14159265358979323846; /* M_PI */

static void rmc_tables(double *c, double *s) {
    for (int i = 0; i < 256; i++) {
        c[i] = cos(2 * i * RMC_PI / 256);
        s[i] = fabs(sin(2 * i * RMC_PI / 256));
    }
}

/* cpu_rotormc.cpp:46-60: h plus cos(neighbour angle) * J, adjacency order. */
static double rmc_field(int var, const uint8_t *st, const double *h, const adjacency *a,
                        const double *cs) {
    double e = h[var];
    for (int k = a->row[var]; k < a->row[var + 1]; k++) e += cs[st[a->col[k]]] * a->w[k];
    return e;
}

/* One run, cpu_rotormc.cpp:104-296.  `stats` receives the state after every
 * beta index divisible by `interval` (interval 0: none). */
static void rmc_run(uint8_t *st, const double *h, const adjacency *a, const double *tf,
                    int spb, int nb, const double *hp, const double *hd, int order,
                    int proposal, const double *cs, const double *sn, uint64_t rng[2],
                    double *de, uint8_t *stats, int interval) {
    const int n = a->n;
    for (int v = 0; v < n; v++) de[v] = rmc_field(v, st, h, a, cs);
    if (proposal <= 1)
        for (int v = 0; v < n; v++) de[v] *= -2 * cs[st[v]];
    for (int i = 0; i < 32; i++) rng_next(rng); /* :141-143 burn-in */
    for (int b = 0; b < nb; b++) {
        const double beta = hp[b], beta_tf = hd[b];
        const double rat = beta_tf / beta;
        for (int sw = 0; sw < spb; sw++) {
            for (int i = 0; i < n; i++) {
                int var = i;
                if (order) var = (int)(rng_next(rng) % (uint64_t)n);
                uint8_t prop = 0;
                double prop_e = 0.0;
                int flip = 0;
                if (proposal == 1) { /* :167-184 */
                    prop = (uint8_t)(128 + st[var]);
                    prop_e = -de[var];
                    if (de[var] <= 0.0) {
                        flip = 1;
                    } else {
                        const uint64_t r = rng_next(rng);
                        if (exp(-de[var] * beta) * RANDMAX_D > (double)r) flip = 1;
                    }
                } else if (proposal == 0) { /* :185-196 */
                    prop = (uint8_t)(128 + st[var]);
                    prop_e = -de[var];
                    const uint64_t r = rng_next(rng);
                    if (RANDMAX_D > (double)r * (1 + exp(de[var] * beta))) flip = 1;
                } else {
                    uint64_t r = rng_next(rng);
                    if (proposal == 2 || rat >= 1) { /* :197-200, 206-207 */
                        prop = (uint8_t)(r % 256);
                    } else { /* :208-233 */
                        const int osi = (int)(rat * 128 - 0.5);
                        const double distc = (osi * (osi + 1)) / (double)(2 * osi + 1);
                        const double p = (rat / 2 * 128 - distc) / (osi + 1 - distc);
                        const uint64_t rl = r;
                        r = rng_next(rng);
                        const uint8_t pac = (p * RANDMAX_D > (double)rl)
                                                ? (uint8_t)((uint64_t)(osi + 1) * (2 * (r % 2) - 1))
                                                : (uint8_t)(r % (uint64_t)(2 * osi + 1) - (uint64_t)osi);
                        prop = (uint8_t)(st[var] + pac);
                    }
                    /* :244-266 */
                    prop_e = rmc_field(var, st, h, a, cs);
                    const double dlm = -beta * prop_e * (cs[prop] - cs[st[var]]) +
                                       beta_tf * tf[var] * (sn[prop] - sn[st[var]]);
                    if (dlm >= 0.0) {
                        flip = 1;
                    } else {
                        const uint64_t r2 = rng_next(rng);
                        if (exp(dlm) * RANDMAX_D > (double)r2) flip = 1;
                    }
                }
                if (flip) { /* :268-287 */
                    if (proposal <= 1) {
                        const double mult = 2 * (cs[st[var]] - cs[prop]);
                        for (int k = a->row[var]; k < a->row[var + 1]; k++) {
                            const int nbv = a->col[k];
                            de[nbv] += mult * a->w[k] * cs[st[nbv]];
                        }
                        de[var] = prop_e;
                    }
                    st[var] = prop;
                }
            }
        }
        if (interval != 0 && b % interval == 0) { /* :289-293 */
            memcpy(stats, st, (size_t)n);
            stats += n;
        }
    }
}

/* cpu_rotormc.cpp:310-326: cos-weighted classical energy. */
static double rmc_energy(int n, const double *h, long m, const int *u, const int *v,
                         const double *J, const uint8_t *st, const double *cs) {
    double e = 0.0;
    for (int i = 0; i < n; i++) e += cs[st[i]] * h[i];
    for (long c = 0; c < m; c++) e += cs[st[u[c]]] * J[c] * cs[st[v[c]]];
    return e;
}

/* Driver, cpu_rotormc.cpp:368-563.  num_seeds 1: one stream across samples
 * (the reference's call); num_seeds == num_samples: sample r as its own call
 * with seed seeds[r].  `stats` holds num_samples blocks of
 * n * (1 + (num_betas - 1) / interval) bytes, one per sample (the reference's
 * own buffer places sample r at r * n * (num_betas / interval); the caller
 * rearranges). */
int rmc_oracle_run(int n, const double *h, long m, const int *u, const int *v,
                   const double *J, const double *tf, int num_samples, uint8_t *states,
                   double *energies, int spb, int nb, const double *hp, const double *hd,
                   const uint64_t *seeds, int num_seeds, int order, int proposal,
                   uint8_t *stats, int interval) {
    if (proposal < 0 || proposal > 3) return ORACLE_EINVAL;
    adjacency a;
    int rc = build_adjacency(&a, n, m, u, v, J);
    if (rc) {
        free_adjacency(&a);
        return rc;
    }
    double cs[256], sn[256];
    rmc_tables(cs, sn);
    double *de = (double *)malloc(sizeof(double) * ((size_t)n + 1));
    if (!de) {
        free_adjacency(&a);
        return ORACLE_ENOMEM;
    }
    const long points = interval ? 1 + (nb - 1) / interval : 0;
    uint64_t rng[2] = {0, 0};
    if (num_seeds == 1) rng_seed(rng, seeds[0]);
    for (int r = 0; r < num_samples; r++) {
        if (num_seeds != 1) rng_seed(rng, seeds[r]);
        uint8_t *st = states + (size_t)r * (size_t)n;
        rmc_run(st, h, &a, tf, spb, nb, hp, hd, order, proposal, cs, sn, rng, de,
                stats ? stats + (size_t)r * (size_t)points * (size_t)n : NULL, stats ? interval : 0);
        energies[r] = rmc_energy(n, h, m, u, v, J, st, cs);
    }
    free(de);
    free_adjacency(&a);
    return num_samples;
}
