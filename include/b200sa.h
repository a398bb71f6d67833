/*
 * b200sa: B200 (sm_100a) simulated-annealing sampler -- C ABI.
 *
 * Drop-in for the simulated-annealing path of dwave-samplers 1.8.0:
 *   C++ core   general_simulated_annealing   dwave/samplers/sa/src/cpu_sa.h:63-78
 *                                             dwave/samplers/sa/src/cpu_sa.cpp:253-362
 *   Cython     simulated_annealing(...)       dwave/samplers/sa/simulated_annealing.pyx:45-50
 *
 * Conventions shared by every entry point
 *   - Plain C types only; no exceptions cross this boundary.  Every function
 *     returns a non-negative value on success and a negative B200SA_E* code on
 *     failure, with a message in `err` (NUL-terminated, truncated to errlen)
 *     when `err` is non-NULL.  The reference throws std::runtime_error through
 *     a nogil Cython call for the same conditions (cpu_sa.cpp:276-279,
 *     302-304), which aborts the process.
 *   - States are int8 spins, row-major num_reads x num_vars, C-contiguous.
 *   - Enumerations keep the reference's numeric values (cpu_sa.h:36-43).
 *   - Seeding.  With num_seeds == num_reads, read r uses its own xorshift128+
 *     stream seeded with seeds[r] and equals a reference call with
 *     num_samples=1, seed=seeds[r].  With num_seeds == 1 the stream is seeded
 *     once and continues across reads exactly as in the reference
 *     (cpu_sa.cpp:283-284, 321-358); that mode runs the reads one after
 *     another on one warp.
 *   - Reentrant: no global mutable state; each call uses its own stream and
 *     device buffers.
 */
#ifndef B200SA_H
#define B200SA_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define B200SA_API __attribute__((visibility("default")))
#else
#define B200SA_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define B200SA_OK 0
#define B200SA_EINVAL (-1)   /* bad argument: lengths, indices, enums */
#define B200SA_ECUDA (-2)    /* CUDA runtime error (message has the detail) */
#define B200SA_ENOMEM (-3)   /* host or device allocation failed */
#define B200SA_ENODEV (-4)   /* no usable sm_100 device */
#define B200SA_ETIMEOUT (-5) /* a bounded device wait expired */
#define B200SA_ERANGE (-6)   /* a fixed capacity was exceeded (call again with more) */

/* cpu_sa.h:36-39 */
#define B200SA_GIBBS 0
#define B200SA_METROPOLIS 1
/* cpu_sa.h:40-43 */
#define B200SA_SEQUENTIAL 0
#define B200SA_RANDOM 1

/* Scheduling modes for the batched entry points. */
#define B200SA_MODE_PERSISTENT 0 /* one launch, device work queue over (problem, read) */
#define B200SA_MODE_PLAIN 1      /* one launch per problem, problems in order */
#define B200SA_MODE_GRAPH 2      /* the persistent launches captured once as a CUDA graph
                                    (plans only; replayed while the buffers are the same) */
#define B200SA_MODE_PLAIN_TUNED 3 /* one launch per problem, each with the autotuned shape
                                     of its size bucket (plain batching with tuned launches) */

/* Replaces the reference's `callback` (cpu_sa.h:61): called between reads,
 * in read order, for each completed read; nonzero stops sampling and the
 * completed prefix is returned (cpu_sa.cpp:357). */
typedef int (*b200sa_interrupt_fn)(void *ctx);

typedef struct {
    int64_t reads;        /* reads completed */
    int64_t attempts;     /* spin-flip attempts: reads x sweeps x num_vars */
    int64_t flips;        /* accepted flips */
    int64_t near_ties;    /* exp() decisions inside the cross-libm tie band */
    int64_t passes;       /* warp passes of the sequential sweep (speculation efficiency) */
    double kernel_ms;     /* device time of the sampling launches (CUDA events) */
    int64_t launches;     /* sweep-kernel launches issued */
    /* Input, optional (NULL: not wanted): a caller-owned host array that
     * receives each completed read's near-tie count, one uint32 per read, in
     * read order (b200sa_sample: num_reads entries; b200sa_sample_batch and
     * b200sa_plan_run: every read of every problem, at the plan's read
     * offsets).  A read with a nonzero count made an exp() decision within
     * 2^-48 of its threshold, where CUDA's exp and the host libm's could
     * decide differently; every other read is bit-exact with the reference.
     * Entries of reads that did not complete are left untouched.  The call
     * keeps this pointer when it resets the counters above. */
    uint32_t *read_near_ties;
} b200sa_stats;

/* One binary quadratic model in Ising form plus its reads.
 * Couplers are COO in input order; that order fixes the adjacency order and
 * the energy summation order exactly as in cpu_sa.cpp:298-316 and :210-227. */
typedef struct {
    int32_t num_vars;
    const double *h;                /* [num_vars] */
    int64_t num_couplers;
    const int32_t *coupler_starts;  /* [num_couplers] */
    const int32_t *coupler_ends;    /* [num_couplers] */
    const double *coupler_weights;  /* [num_couplers] */
    int32_t num_reads;
    int8_t *states;                 /* [num_reads * num_vars], in/out */
    double *energies;               /* [num_reads], out */
    int32_t sweeps_per_beta;
    int32_t num_betas;
    const double *beta_schedule;    /* [num_betas] */
    const uint64_t *seeds;          /* [num_reads] per-read seeds */
    int32_t varorder;               /* B200SA_SEQUENTIAL / B200SA_RANDOM */
    int32_t proposal;               /* B200SA_GIBBS / B200SA_METROPOLIS */
} b200sa_problem;

/* Replaces general_simulated_annealing (cpu_sa.h:63-78, cpu_sa.cpp:253-362)
 * behind simulated_annealing.pyx:172-186.  Host buffers; `states` is
 * overwritten in place for the reads completed.  Returns the number of reads
 * completed (num_reads unless interrupted) or a negative error. */
B200SA_API int b200sa_sample(int32_t num_vars, const double *h, int64_t num_couplers,
                  const int32_t *coupler_starts, const int32_t *coupler_ends,
                  const double *coupler_weights, int32_t num_reads,
                  int8_t *states, double *energies, int32_t sweeps_per_beta,
                  int32_t num_betas, const double *beta_schedule,
                  const uint64_t *seeds, int32_t num_seeds, int32_t varorder,
                  int32_t proposal, b200sa_interrupt_fn interrupt_fn,
                  void *interrupt_ctx, int32_t device, b200sa_stats *stats,
                  char *err, size_t errlen);

/* Many independent problems (uneven sizes, read counts and schedules), host
 * buffers.  The reference has no batched entry point; each problem's reads
 * equal the per-read reference calls.  mode: B200SA_MODE_*.  When the
 * environment variable B200SA_TUNE_CACHE names a file, persistent and graph
 * runs use the autotuner's choices from it (measuring buckets it lacks; see
 * b200sa_plan_autotune).
 * Returns the total number of reads completed or a negative error. */
B200SA_API int b200sa_sample_batch(const b200sa_problem *problems, int32_t num_problems,
                        int32_t mode, int32_t device, b200sa_stats *stats,
                        char *err, size_t errlen);

/* ---- Device-resident plans (inputs kept in HBM across runs) --------------
 * A plan packs the problems (order-preserving CSR, schedules, seeds) once and
 * keeps them on the device.  Runs take DEVICE pointers for the states, laid
 * out problem after problem (see b200sa_plan_layout).  No reference
 * counterpart: this is the resident form of b200sa_sample_batch. */
typedef struct b200sa_plan_s *b200sa_plan;

B200SA_API int b200sa_plan_create(const b200sa_problem *problems, int32_t num_problems,
                       int32_t device, b200sa_plan *out, char *err,
                       size_t errlen);

/* Per-problem element offsets into the concatenated state array (int8) and
 * read offsets into the energy / seed arrays; each array has num_problems+1
 * entries (the last is the total). */
B200SA_API int b200sa_plan_layout(b200sa_plan plan, int64_t *state_offsets,
                       int64_t *read_offsets);

/* Anneal on the device.  d_states_in may equal d_states_out.  d_seeds may be
 * NULL (the seeds given at plan creation are used).  `stream` is a
 * cudaStream_t; NULL selects the plan's own stream (pass cudaStreamLegacy for
 * the legacy default stream).  The call returns after the
 * work is enqueued when `sync` is 0, and after it completes when 1 (stats
 * are filled only when sync is 1).  Runs of one plan must not overlap in time
 * (they share the plan's queue heads, counters and global slots). */
B200SA_API int b200sa_plan_run(b200sa_plan plan, int32_t mode, const int8_t *d_states_in,
                    int8_t *d_states_out, double *d_energies,
                    const uint64_t *d_seeds, void *stream, int32_t sync,
                    b200sa_stats *stats, char *err, size_t errlen);

B200SA_API int b200sa_plan_destroy(b200sa_plan plan);

/* Replaces the fields h[num_vars] and coupler weights J[num_couplers] (host
 * arrays, COO order as at creation) of problem `problem`; couplers, schedule
 * and seeds are kept, and so is a captured graph.  Waits for the plan's last
 * run and returns when the device copy is updated.  No reference counterpart:
 * for learning loops that re-sample the same models with new parameters. */
B200SA_API int b200sa_plan_set_weights(b200sa_plan plan, int32_t problem, const double *h,
                                       const double *J, char *err, size_t errlen);

/* Device-side form of b200sa_plan_set_weights for every problem of the plan
 * at once (no reference counterpart): d_h holds the fields of all problems
 * concatenated (problem after problem, num_vars each) and d_J their coupler
 * weights (num_couplers each, COO order as at creation), both DEVICE arrays.
 * The update is enqueued on `stream` (a cudaStream_t; NULL selects the
 * plan's own stream): runs enqueued before it on that stream see the old
 * weights, runs after it the new ones; a captured graph stays valid.  The
 * first call builds the scatter map on the device (it allocates and waits);
 * later calls launch one kernel and return at once.  Returns 0 or a negative
 * error. */
B200SA_API int b200sa_plan_set_weights_device(b200sa_plan plan, const double *d_h,
                                              const double *d_J, void *stream, char *err,
                                              size_t errlen);

/* ---- Autotuner (no reference counterpart) ---------------------------------
 * For every non-empty bucket of a plan (size class x acceptance rule x order)
 * times candidate launch configurations -- warps per CTA, CTAs per SM, the
 * kernel's register budget (128, 80 or 64 registers a thread: fewer spill
 * more but let more reads run per SM), and where delta energies and spins live
 * (shared memory, a global slot, or spins shared and energies global) -- on a
 * sample
 * of the bucket's reads (its largest problems, 8 betas spread over each
 * schedule) and keeps the fastest for the plan's persistent and graph runs.
 * Every configuration computes the same results; only speed changes.  The
 * choices are cached in the text file `cache_path` (NULL: no file), keyed by
 * GPU, library version, kind, size and mean degree, and reused unless flags
 * has B200SA_TUNE_FORCE.  Writes up to report_cap entries and returns the
 * number of non-empty buckets, or a negative error. */
#define B200SA_TUNE_FORCE 1
typedef struct {
    int32_t bucket;
    int32_t kind;           /* bit 0 Gibbs, bit 1 random order, bit 2 in-window resolution */
    int32_t max_n;
    int64_t items;          /* reads in the bucket */
    int32_t staging;        /* state: 0 global slot (L2), 1 shared memory, 2 spins in
                               shared memory and delta energies in the global slot, 3 spins
                               and a band of delta energies around the window in shared
                               memory, the rest in the global slot (banded problems) */
    int32_t warps_per_cta;
    int32_t ctas_per_sm;
    int32_t registers;      /* register budget per thread of the chosen kernel */
    double attempts_per_s;  /* measured on the sample */
    int32_t from_cache;
    int32_t candidates;     /* configurations measured (0 when cached) */
} b200sa_tune_entry;

B200SA_API int b200sa_plan_autotune(b200sa_plan plan, const char *cache_path, int32_t flags,
                                    b200sa_tune_entry *report, int32_t report_cap, char *err,
                                    size_t errlen);

/* Per-bucket figures of a plan's last persistent or graph run (no reference
 * counterpart).  Buckets group the reads by size class and kernel kind; each
 * is one launch.  ms is that launch's device time (CUDA events on the
 * bucket's stream, captured into the graph in graph mode; -1 when unknown),
 * model_bytes the bytes the sweep's state accesses amount to (per read: the
 * initial delta energies n(8 + 13d), 9 per attempt, 29d + 9 per flip and
 * the final energy 9n + 14m, d the mean list length), most of them served
 * from shared memory, L1 and L2.  Waits for the run.  Returns the number of
 * non-empty buckets (up to cap entries written) or a negative error. */
typedef struct {
    int32_t bucket;
    int32_t kind;           /* bit 0 Gibbs, bit 1 random order, bit 2 in-window resolution */
    int32_t max_n;
    int64_t reads;
    int64_t attempts;
    int64_t flips;
    int64_t passes;
    double model_bytes;
    double ms;
    int32_t staging;        /* state location of the launch (see b200sa_tune_entry) */
    int32_t warps_per_cta;
    int32_t grid;
    int32_t registers;
} b200sa_bucket_report;

B200SA_API int b200sa_plan_bucket_report(b200sa_plan plan, b200sa_bucket_report *out,
                                         int32_t cap, char *err, size_t errlen);

/* ---- Steepest descent ---------------------------------------------------------
 * Replaces steepest_gradient_descent (dwave/samplers/greedy/src/descent.cpp:
 * 315-405, descent.h; bound by dwave/samplers/greedy/descent.pyx:22-112): every
 * sample descends from its row of `states` (host, num_samples x num_vars int8,
 * overwritten) by flipping the variable with the most negative flip energy
 * (ties to the lower index) until none is negative; energies[r] and
 * num_steps[r] receive its energy and number of flips.  large_sparse_opt
 * selects the update order of the reference's ordered-set solver (same
 * selection; neighbours updated with the spin before the flip).  A sample
 * stops after max_steps flips (0: 1000 * num_vars + 10^6): a self-loop of
 * positive weight, or spins other than +-1, can make descent cycle (the
 * reference then never returns); the call then returns B200SA_ETIMEOUT with
 * the states reached and num_steps == max_steps for those samples.  Returns
 * num_samples or a negative error. */
B200SA_API int b200sa_steepest_descent(int32_t num_vars, const double *h, int64_t num_couplers,
                                       const int32_t *coupler_starts,
                                       const int32_t *coupler_ends,
                                       const double *coupler_weights, int32_t num_samples,
                                       int8_t *states, double *energies, uint32_t *num_steps,
                                       int32_t large_sparse_opt, uint32_t max_steps,
                                       int32_t device, char *err, size_t errlen);

/* ---- Rotor-model annealing (SQA) -------------------------------------------
 * Replaces general_simulated_annealing of the rotor Monte Carlo
 * (dwave/samplers/sqa/src/cpu_rotormc.cpp:368-563, cpu_rotormc.h; bound at
 * dwave/samplers/sqa/rotormc_annealing.pyx:54-236).  States are uint8 angles
 * (theta = 2*pi*index/256), host arrays, num_samples x num_vars, overwritten.
 * hp_field / hd_field: num_betas problem and driver inverse temperatures;
 * trans_fields: num_vars transverse fields.  proposal: 0 GibbsNonErgodic,
 * 1 MetropolisNonErgodic, 2 MetropolisUniform, 3 MetropolisTF (the
 * reference's enum order).  seeds: num_seeds == 1 continues one stream over
 * the samples exactly as one reference call (samples then run one after
 * another); num_seeds == num_samples makes sample r equal a reference call
 * with num_samples = 1 and seed = seeds[r] (samples run in parallel).
 * statistics (NULL: none) receives, for schedule_sample_interval > 0, the
 * state after every beta index divisible by the interval: num_samples blocks
 * of num_vars * (1 + (num_betas - 1) / interval) bytes, laid out as the
 * reference's call lays them out (with one stream, sample r's block starts at
 * r * num_vars * (num_betas / interval)).  near_ties (optional) counts
 * exp() decisions within 2^-48 of the threshold (expected 0).  Returns
 * num_samples or a negative error. */
B200SA_API int b200sa_rotor_anneal(int32_t num_vars, const double *h, int64_t num_couplers,
                                   const int32_t *coupler_starts, const int32_t *coupler_ends,
                                   const double *coupler_weights, const double *trans_fields,
                                   int32_t num_samples, uint8_t *states, double *energies,
                                   int32_t sweeps_per_beta, int32_t num_betas,
                                   const double *hp_field, const double *hd_field,
                                   const uint64_t *seeds, int32_t num_seeds,
                                   int32_t randomize_order, int32_t proposal,
                                   uint8_t *statistics, int32_t schedule_sample_interval,
                                   int32_t device, int64_t *near_ties, char *err,
                                   size_t errlen);

/* ---- Path-integral Monte Carlo annealing (SQA) ----------------------------
 * Replaces general_simulated_annealing of localPIMC
 * (dwave/samplers/sqa/src/localPIMC.cpp:585-715, localPIMC.h:55-81; bound at
 * dwave/samplers/sqa/pimc_annealing.pyx:45-283).  A sample is a set of world
 * lines over 2^16 Trotter slices: the first slice (states, int8 +-1, host,
 * num_samples x num_vars, overwritten) and, per variable, the slices where
 * its spin flips (its breaks).  hp_field / hd_field: num_betas inverse
 * temperatures (invTemp) and transverse fields (Gamma); every schedule step
 * makes sweeps_per_beta * num_vars updates of uniformly drawn qubits
 * (qubits_per_update == 1) or of chains of qubits_per_chain consecutive
 * variables (any other value; Swendsen-Wang joins with
 * chain_coupler_strength).  seeds: num_seeds == 1 continues one mt19937 stream
 * over the samples exactly as one reference call; num_seeds == num_samples
 * makes sample r equal a reference call with num_samples = 1 and seed =
 * seeds[r] (samples run in parallel).  A seed of 0 (the reference's
 * nondeterministic generator) draws a nonzero seed from std::random_device.
 * project_inputs == 0: sample r starts from num_breaks[r][v] positions per
 * variable read in order from breaks_in (breaks_in_size entries).
 * project_outputs == 0: num_breaks receives the final counts and breaks_out
 * (breaks_out_size entries) the positions, filled as the reference's
 * readBreaks fills its buffer (localPIMC.cpp:185-200).  statistics receives,
 * for schedule_sample_interval > 0, the first slice after every schedule
 * index divisible by the interval (num_samples x points x num_vars, points =
 * 1 + (num_betas - 1) / interval).  break_capacity bounds the breaks of a
 * variable and the proposals of one update (0: from the largest Gamma);
 * exceeding it returns B200SA_ERANGE.  near_ties (optional) counts log / tanh
 * / exp decisions within 2^-48 of their threshold (expected 0).  Returns
 * num_samples or a negative error. */
B200SA_API int b200sa_path_anneal(
    int32_t num_vars, const double *h, int64_t num_couplers, const int32_t *coupler_starts,
    const int32_t *coupler_ends, const double *coupler_weights, int32_t num_samples,
    int8_t *states, double *energies, int32_t sweeps_per_beta, int32_t num_betas,
    const double *hp_field, const double *hd_field, double chain_coupler_strength,
    int32_t qubits_per_chain, int32_t qubits_per_update, const uint32_t *seeds,
    int32_t num_seeds, int32_t project_inputs, int32_t project_outputs, int32_t *num_breaks,
    const int32_t *breaks_in, int64_t breaks_in_size, int32_t *breaks_out,
    int64_t breaks_out_size, int8_t *statistics, int32_t schedule_sample_interval,
    int32_t break_capacity, int32_t device, int64_t *near_ties, char *err, size_t errlen);

/* ---- Sample moments (no reference counterpart) ------------------------------
 * For the gradient of log Z of p(s) ~ exp(-beta*E(s)), E as in cpu_sa.cpp:210-227:
 * d log Z/d h_i = -beta <s_i>, d log Z/d J_c = -beta <s_u(c) s_v(c)>.  Adds the
 * exact integer sums over reads of s_i (sum_s) and of s_u*s_v per coupler in COO
 * order (sum_ss) to the caller's zero-initialised device arrays, for many
 * problems in one launch.  All pointers are device memory; coupler indices
 * must be valid (num_vars <= 4096). */
typedef struct {
    int32_t num_vars;
    int64_t num_couplers;
    int32_t num_reads;
    const int8_t *states;           /* [num_reads * num_vars] */
    const int32_t *coupler_starts;  /* [num_couplers] */
    const int32_t *coupler_ends;    /* [num_couplers] */
    int64_t *sum_s;                 /* [num_vars], accumulated into */
    int64_t *sum_ss;                /* [num_couplers], accumulated into */
} b200sa_moments_problem;

B200SA_API int b200sa_edge_moments(const b200sa_moments_problem *problems, int32_t num_problems,
                                   int32_t device, void *stream, char *err, size_t errlen);

/* No counterpart in the reference.  Writes num_reads x num_vars uniform +-1
 * initial states (reads read0 .. read0+num_reads-1 of model model_index) to
 * device memory as a counter-based hash of (init_seed, model, read, variable),
 * so that any range of reads can be regenerated identically (samples are
 * recomputed from their seeds instead of stored).  Asynchronous on `stream`
 * (a cudaStream_t; NULL = legacy default stream).  Returns 0 or a negative
 * error. */
B200SA_API int b200sa_random_states(uint64_t init_seed, uint64_t model_index, int64_t read0,
                                    int64_t num_reads, int32_t num_vars, int8_t *d_states,
                                    int32_t device, void *stream, char *err, size_t errlen);

/* No counterpart in the reference.  The sampler for callers that cannot
 * allocate device memory while they run (all device memory owned by a
 * pre-sized pool or arena, plugin hosts that allow allocation only at
 * start-up, loops where cudaMalloc/cudaFree and their implicit device-wide
 * synchronization are not acceptable).  Every pointer is DEVICE memory owned
 * by the caller: inputs h, couplers, beta schedule, per-read seeds and initial
 * states; outputs final states and energies.  The call allocates nothing: its
 * working memory is one fixed 4 MiB array inside the library, held on each
 * device that loads the library until the process exits, which limits the
 * problem to num_vars <= 4096, num_couplers <= 65536, num_betas <= 16384 and
 * num_reads <= 16384 (larger problems return B200SA_EINVAL).  Per-read seeds
 * only (read r equals a reference call with num_samples=1, seed=seeds[r]).
 * All calls on a device share that array: calls that overlap on the GPU race
 * and must be serialized by the caller.  The first call on a device sets the
 * array up (device address, RNG tables, device properties).  `stream` is a
 * cudaStream_t (NULL = legacy default stream); the call returns when the work
 * is complete, so it cannot be recorded into a CUDA graph (a call on a
 * capturing stream returns B200SA_EINVAL).  Near ties: d_read_near_ties
 * (optional DEVICE array, num_reads entries) receives each read's count of
 * exp() decisions within 2^-48 of their threshold, and near_ties (optional
 * host pointer) their total; a read with a nonzero count may differ from the
 * reference, every other read is bit-exact.  Returns num_reads or a negative
 * error. */
B200SA_API int b200sa_sample_noalloc(
    int32_t num_vars, const double *d_h, int64_t num_couplers, const int32_t *d_coupler_starts,
    const int32_t *d_coupler_ends, const double *d_coupler_weights, int32_t num_reads,
    const int8_t *d_states_in, int8_t *d_states_out, double *d_energies,
    int32_t sweeps_per_beta, int32_t num_betas, const double *d_beta_schedule,
    const uint64_t *d_seeds, int32_t varorder, int32_t proposal, int32_t device, void *stream,
    uint32_t *d_read_near_ties, int64_t *near_ties, char *err, size_t errlen);

/* Diagnostic, no reference counterpart: checks on the device that the
 * single-precision acceptance bounds used before the exact double-precision
 * test never disagree with it.  counts[6] = Metropolis {samples, decided by
 * the bounds, disagreements}, Gibbs {samples, decided by the bounds,
 * disagreements}; both disagreement counts must be 0. */
B200SA_API int b200sa_check_acceptance(int64_t samples, uint64_t seed, int32_t device,
                                       int64_t counts[6], char *err, size_t errlen);

/* Version string of this library. */
B200SA_API const char *b200sa_version(void);

#ifdef __cplusplus
}
#endif

#endif /* B200SA_H */
