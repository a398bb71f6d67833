// Types shared by the host packer, the launch code and the sm_100a kernels.
#pragma once
#include <cstdint>

namespace b200sa {

// RNG output ring per read (shared memory).  The ring holds the next
// kRing outputs of the read's xorshift128+ stream; it is refilled one half at
// a time, each lane producing kPerLane consecutive outputs from its own
// segment-start state, and each lane then jumps that state kHalf steps ahead
// with a precomputed GF(2) matrix (xorshift128+ is linear over GF(2)).
constexpr int kRing = 512;
constexpr int kHalf = kRing / 2;
constexpr int kPerLane = kHalf / 32;

// vinfo byte per variable:
//   bits 0-5: distance to the nearest later neighbour (u - v for the smallest
//             neighbour u > v), capped at 32.  A flip of v can only change the
//             decision of a variable inside the current 32-wide window if
//             that variable is at least this far ahead.
//   bit 6   : v's adjacency list names some target more than once (self-loop
//             or repeated coupler), so its updates must run one at a time to
//             keep the reference's order of additions to the same slot.
constexpr uint8_t kDistMask = 0x3f;
constexpr uint8_t kDupFlag = 0x40;

struct ProblemDev {
    int32_t n;
    int32_t sweeps_per_beta;
    int32_t num_betas;
    int32_t num_reads;
    int64_t m;              // couplers
    int64_t state_offset;   // element offset of read 0 in the state arrays
    int64_t read_offset;    // offset of read 0 in energies / seeds / stats
    const int32_t *row;     // [n+1] adjacency offsets
    const int32_t *col;     // [2m] neighbour index, coupler input order
    const double *w;        // [2m] coupling
    const double *h;        // [n]
    const uint8_t *vinfo;   // [n]
    const int32_t *cu;      // [m] COO, input order (energy)
    const int32_t *cv;      // [m]
    const double *cw;       // [m]
    const double *betas;    // [num_betas]
    const double *thresholds;  // [num_betas] 44.36142 / beta, host-divided
    int32_t varorder;       // 0 sequential, 1 random
    int32_t proposal;       // 0 Gibbs, 1 Metropolis
};

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
};

// Shared-stream carry layout (uint64 words).
constexpr int kCarryLaneWords = 64;                 // 32 lanes x 2 words
constexpr int kCarryWords = kRing + kCarryLaneWords + 2;  // ring, lanes, q, base

}  // namespace b200sa
