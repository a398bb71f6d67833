// Types shared by the host packer, the launch code and the sm_100a kernels.
#pragma once
#include <cstdint>

#include <vector_types.h>

namespace b200sa {

// RNG output ring per read (shared memory).  The ring holds the next
// kRing outputs of the read's xorshift128+ stream; it is refilled one half at
// a time, each lane producing kPerLane consecutive outputs from its own
// segment-start state, and each lane then jumps that state kHalf steps ahead
// with a precomputed GF(2) matrix (xorshift128+ is linear over GF(2)).
constexpr int kRing = 256;
constexpr int kHalf = kRing / 2;
constexpr int kPerLane = kHalf / 32;

// Per-variable adjacency record (uint2): x = start of the variable's list,
// y = its degree (list length).
constexpr uint32_t kDegMask = 0x00ffffffu;
constexpr uint32_t kMaxDegree = kDegMask;

// Speculation arrays, read once per variable and pass (kept as two compact
// arrays, 5 bytes per variable, so they stay in the L1 left beside the
// shared regions):
//   dist:  distance to the nearest later neighbour (u - v for the smallest
//          neighbour u > v), capped at kDistCap.  A flip of v can only change
//          the decision of a later variable of the current window if that
//          variable is at least this far ahead.
//   share: conflict mask.  Bit 0 is set when v's list names a target twice;
//          bit j (1..31) when v and v + j have a common neighbour.  Two
//          committed flips can add into the same delta-energy slot only
//          through one of these.
constexpr uint32_t kDistCap = 32;  // the speculative window

struct ProblemDev {
    int32_t n;
    int32_t sweeps_per_beta;
    int32_t num_betas;
    int32_t num_reads;
    int64_t m;              // couplers
    int64_t state_offset;   // element offset of read 0 in the state arrays
    int64_t read_offset;    // offset of read 0 in energies / seeds / stats
    const uint2 *vinfo;     // [n] adjacency record (see above)
    const uint8_t *dist;    // [n] speculation distance (see above)
    const uint32_t *share;  // [n] conflict mask (see above)
    const int32_t *col;     // [2m] neighbour index, coupler input order
    const double *w;        // [2m] coupling
    const double *h;        // [n]
    const int32_t *cu;      // [m] COO, input order (energy)
    const int32_t *cv;      // [m]
    const double *cw;       // [m]
    const double *betas;    // [num_betas]
    const double *thresholds;  // [num_betas] 44.36142 / beta, host-divided
    int32_t varorder;       // 0 sequential, 1 random
    int32_t proposal;       // 0 Gibbs, 1 Metropolis
    // Every adjacency list has this length (1..32) and list v starts at
    // v * regular_degree; 0 when the lists differ in length.
    int32_t regular_degree;
    uint32_t regular_magic;  // ceil(2^16 / regular_degree): t / D == (t * magic) >> 16 for t < 1024
    // In-window resolution of the sequential sweep (1: on, for reads whose
    // spins are all +-1).  back[v] = {mask, start}: bit o (1..31) of mask set
    // when v - o is a neighbour of v; bw[start ..] the couplings of those
    // neighbours, offsets descending (the order the reference adds their
    // flips' contributions).  No list may name a target twice.
    int32_t resolve;
    // Dense updates (1: on; needs resolve): the committed flips' contributions
    // are pulled by each variable's owner lane, flip after flip, from
    // dense_w[j*n + x] (the coupling of j and x) where bit x of
    // dense_bits[4j ..] is set.  n <= kDenseMaxN.
    int32_t dense;
    const uint2 *back;
    const double *bw;
    const double *dense_w;
    const uint32_t *dense_bits;
    // Banded delta energies (kStageBand): adjacency entries mostly within
    // band_b of their variable; band_w is the shared-memory ring size (a power
    // of two >= 2 band_b + 128), 0 when the problem is not banded.
    int32_t band_b;
    int32_t band_w;
};
constexpr int kDenseMaxN = 128;
constexpr int kBandMaxSlots = 8192;  // 64 KB of delta energies per warp at most

// Per-read counters written by the kernel.
struct ReadStats {
    unsigned long long flips;
    unsigned long long passes;
    unsigned int near_ties;
    unsigned int pad;
};

struct LaunchArgs {
    const ProblemDev *problems;
    const int64_t *items;          // (problem << 32) | read, execution order
    int64_t num_items;
    unsigned long long *queue_head;  // persistent mode work-queue head (nullptr: static)
    const int8_t *states_in;
    int8_t *states_out;
    double *energies;
    const uint64_t *seeds;         // indexed by read_offset + r
    ReadStats *stats;              // indexed by read_offset + r
    int32_t shared_stream;         // 1: one warp, items in order, one RNG stream
    uint64_t *rng_carry;           // shared-stream state between launches
    int32_t carry_in;              // 1: resume the stream from rng_carry
    int32_t smem_cap_n;            // largest n kept in the warp's shared region
    double *scratch_de;            // global fallback state, one slot per warp
    int8_t *scratch_s;
    int64_t scratch_stride;        // elements per slot
    int64_t num_slots;
    // Random order: bytes of the per-warp bitmap of variables touched by the
    // window's accepted flips (touch_bytes_for of the launch's largest n), in
    // the shared region between the scratch and the state; 0 otherwise.
    int32_t touch_bytes;
    // kStageBand: slots of the per-warp delta-energy band (0 otherwise).
    int32_t band_cap;
};

// Arguments of the steepest-descent kernel (sd_kernel.cuh): one problem,
// items (0 << 32) | sample taken from a queue head.
struct SdArgs {
    const ProblemDev *problem;
    const int64_t *items;        // (0 << 32) | sample
    int64_t num_items;
    unsigned long long *queue_head;
    const int8_t *states_in;
    int8_t *states_out;
    double *energies;
    uint32_t *steps;
    uint32_t max_steps;
    int32_t smem_cap_n;          // state in shared memory when > 0
    double *scratch_fe;          // else per-warp global slots
    int8_t *scratch_s;
    int64_t scratch_stride;
    unsigned long long *capped;  // samples stopped by max_steps
};

// Per-warp shared region of the descent kernel: 32 doubles for equal-target
// sums, then (state in shared memory) flip energies and spins.
constexpr int kSdScratchBytes = 32 * 8;  // equal-target sums
inline int sd_region_bytes(int cap_n) {
    return kSdScratchBytes + cap_n * 8 + ((cap_n + 15) & ~15);
}

// Arguments of the rotor-model annealing kernel (rmc_kernel.cuh).
struct RmcArgs {
    int32_t n;
    int64_t m;
    const uint2 *vinfo;      // [n] {list start, degree}
    const int32_t *col;      // adjacency, coupler input order
    const double *w;
    const double *h;
    const double *tf;        // [n] transverse fields
    const int32_t *cu, *cv;  // COO (energy order)
    const double *cw;
    const double *hp, *hd;   // [num_betas] problem and driver field schedules
    int32_t num_betas;
    int32_t sweeps_per_beta;
    const uint64_t *seeds;
    int32_t shared_stream;   // 1: one thread, samples in order, one RNG stream
    int32_t num_samples;
    uint8_t *rows;           // [num_samples][n] initial states in, final states out
    uint8_t *states;         // working copy, interleaved: element (v, r) at v * num_samples + r
    double *de;              // interleaved like states
    double *energies;
    uint8_t *stats;          // [num_samples][points][n], or null
    int32_t interval;
    const double *cos_table, *sin_table;  // [256]
    unsigned long long *near;
};

// Arguments of the path-integral Monte Carlo kernel (pimc_kernel.cuh).  One
// thread per sample (a "slot"); every slot owns an mt19937 state and a
// scratch area in global memory.  Break lists have a fixed capacity per
// variable; proposals and domains per update have one too.
struct PimcArgs {
    int32_t n;
    int64_t m;
    const uint2 *vinfo;      // [n] {list start, degree}
    const int32_t *col;      // adjacency, coupler input order
    const double *w;
    const double *h;
    const int32_t *cu, *cv;  // COO (energy order)
    const double *cw;
    const double *hp, *hd;   // [num_betas] problem (invTemp) and driver (Gamma) schedules
    int32_t num_betas;
    int32_t sweeps_per_beta;
    double jchain;           // chain coupling (Swendsen-Wang joins)
    int32_t qpc;             // qubits per chain (chain update)
    int32_t chains;          // n / qpc
    const uint32_t *seeds;
    int32_t shared_stream;   // 1: one thread, samples in order, one generator
    int32_t num_samples;
    int8_t *states;          // [num_samples][n], the first Trotter slice
    int32_t *counts;         // [num_samples][n] breaks per variable
    int32_t *breaks;         // [num_samples][n][cap_breaks]
    int32_t cap_breaks;
    int32_t cap_props;       // proposals per qubit and update
    uint32_t *mt;            // [slots][kMtWords]
    int32_t *scratch_i;      // [slots][scratch_ints]
    double *scratch_d;       // [slots][scratch_doubles]
    int64_t scratch_ints, scratch_doubles;
    double *energies;
    int8_t *stats;           // [num_samples][points][n], or null
    int32_t interval;
    unsigned long long *near;
    int32_t *overflow;       // set when a capacity would be exceeded
};
constexpr int kMtWords = 624;

// Nibble tables of the RNG jump matrix: entry [k][v] is the jump applied to
// the state whose only set bits are the nibble value v at nibble position k.
constexpr int kJumpNibbles = 32;
constexpr int kJumpTable = kJumpNibbles * 16;

// Shared-stream carry layout (uint64 words).
constexpr int kCarryLaneWords = 64;                 // 32 lanes x 2 words
constexpr int kCarryWords = kRing + kCarryLaneWords + 2;  // ring, lanes, q, base

// Per-warp shared region: RNG ring, scratch (32 doubles for equal-slot sums,
// 32 ints for the rank table of accepted flips; then the lanes' RNG
// segment-start states and the read's counters, which the sweep loop keeps
// out of registers), delta energies, spins.  (region_bytes_for keeps every
// region a multiple of 16 bytes.)
constexpr int kScratchHotBytes = 32 * 8 + 32 * 4;
constexpr int kColdBytes = 32 * 16 + 32;
constexpr int kScratchBytes = kScratchHotBytes + kColdBytes;
inline int region_bytes_for(int cap_n) {
    const int spins = (cap_n + 15) & ~15;
    return kRing * 8 + kScratchBytes + ((cap_n * 8 + 15) & ~15) + spins;
}

// Where a read's state lives: kStageGlobal keeps delta energies and spins in
// a per-warp global slot (L2-resident), kStageShared both in the warp's
// shared region, kStageSpins the spins in the shared region and the delta
// energies in the global slot (a smaller global footprint, and the spin
// reads of the neighbour updates stay on chip).
constexpr int kStageGlobal = 0;
constexpr int kStageShared = 1;
constexpr int kStageSpins = 2;
// kStageBand: spins in the shared region, the delta energies of a band of
// variables around the window in a shared-memory ring after them (band_cap
// slots), the others in the global slot (sequential order, banded problems).
constexpr int kStageBand = 3;
constexpr int kNumStages = 4;
inline int region_bytes_for_stage(int stage, int cap_n, int band_cap = 0) {
    if (stage == kStageShared) return region_bytes_for(cap_n);
    if (stage == kStageSpins) return kRing * 8 + kScratchBytes + ((cap_n + 15) & ~15);
    if (stage == kStageBand) return kRing * 8 + kScratchBytes + ((cap_n + 15) & ~15) + 8 * band_cap;
    return kRing * 8 + kScratchBytes;
}

// Random order keeps a bitmap of n bits per warp (16-byte multiple).
inline int touch_bytes_for(bool random_order, int max_n) {
    return random_order ? (((max_n + 31) / 32) * 4 + 15) & ~15 : 0;
}

}  // namespace b200sa
