// Host-side packing of one Ising problem into the device layout.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "b200sa.h"

namespace b200sa {

struct PackedAdjacency {
    std::vector<int32_t> row;     // n+1
    std::vector<int32_t> col;     // 2m
    std::vector<double> w;        // 2m
    std::vector<uint32_t> vinfo;  // 2n: per variable {list start, degree}
    std::vector<uint8_t> dist;    // n: speculation distance (ProblemDev::dist)
    std::vector<uint32_t> share;  // n: conflict mask (ProblemDev::share)
    int32_t max_degree = 0;
    int32_t regular_degree = 0;   // common list length when all lists are equally long
    bool any_dup = false;         // some list names a target twice (self-loop / repeat)
    // In-window resolution (ProblemDev::back, ProblemDev::bw): per variable v
    // {mask of offsets o in 1..31 with v - o a neighbour, start in bw}; bw the
    // couplings of those neighbours, nearest-last (offsets descending), and
    // bw_src the adjacency entry each coupling comes from.
    std::vector<uint32_t> back;   // 2n
    std::vector<double> bw;
    std::vector<int32_t> bw_src;
    bool resolve = false;         // in-window resolution enabled (ProblemDev::resolve)
    // Dense updates (ProblemDev::dense): n <= 128, average degree >= n/8, no
    // repeated targets.  dense_w[j*n + x] is the coupling of j and x (0 when
    // they are not neighbours) and dense_bits[4j .. 4j+3] the 128-bit mask of
    // j's neighbours.
    std::vector<double> dense_w;
    std::vector<uint32_t> dense_bits;
    bool dense = false;
    // Banded delta energies (ProblemDev::band_b / band_w): the smallest
    // offset b >= 32 that covers 97% of the adjacency entries, and the ring
    // size (power of two >= 2b + 128, at most kBandMaxSlots, at most half of
    // n); band_w 0 when the problem is not banded.
    int32_t band_b = 0;
    int32_t band_w = 0;
};

// Validates one problem's arguments (lengths, indices, enums, degree limit).
// Returns B200SA_OK or B200SA_EINVAL with a message.
int validate_problem(const b200sa_problem &p, std::string &msg);

// Order-preserving adjacency, same order as cpu_sa.cpp:298-316.
void pack_adjacency(const b200sa_problem &p, PackedAdjacency &out);

// Columns of the GF(2) matrix that advances an xorshift128+ state by `steps`
// steps: column b is the state reached from the unit state with only bit b
// set (bits 0-63 = word 0, 64-127 = word 1).  Four uint32 words per column:
// word0 lo, word0 hi, word1 lo, word1 hi.
void rng_jump_columns(int64_t steps, uint32_t out[128][4]);

// Nibble tables of that matrix: out[k*16 + v] (four words each) is the XOR of
// the columns selected by the bits of v at nibble position k.
void rng_jump_nibbles(const uint32_t cols[128][4], uint32_t out[][4]);

}  // namespace b200sa
