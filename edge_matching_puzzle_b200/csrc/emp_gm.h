// Glutton max search on the GPU (emp_gm.cu): launch interface.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace emp {

// Device-side search state, one per search (global memory).
struct GmState {
    uint32_t level;              // pieces placed (the reference's m_level)
    uint32_t max;                // best level reached (m_max)
    int32_t status;              // 0 full board, 1 budget or deadline reached, 2 search exhausted,
                                 // 3 multi-block search stopped by a barrier timeout
    uint32_t new_level;          // the kernel loop's l_new_level
    uint32_t pop_index;          // info index returned by the last pop
    uint32_t pad[3];
    unsigned long long trials;   // candidate trial evaluations (every pass)
    unsigned long long pushes;   // committed placements
    unsigned long long pops;
    unsigned long long passes;   // validity passes
    unsigned long long levels;   // levels evaluated
    uint32_t position_index[256];
    uint32_t info_index[256];
    uint32_t played[256];        // (o<<16) | (piece<<8) | position
    uint32_t max_played[256];
    uint32_t avail[8];           // piece availability bits
};

// Exchange area of the multi-block search (one per search, global memory).
constexpr uint32_t kMaxGridBlocks = 256;
struct GmGrid {
    uint32_t bar_count, bar_gen;  // grid barrier
    int error;                    // a barrier wait ran out of time
    uint32_t stop;                // block 0's decision at the top of a level
    uint32_t any_invalid[3];      // per pass buffer (pass number mod 3)
    uint32_t next_info[3];
    uint32_t inval[3][256][32];
    unsigned long long blk_key[3][kMaxGridBlocks];
    uint32_t blk_order[3][kMaxGridBlocks];
};

struct GmLaunch {
    const uint8_t* pieces;       // [256][4] colours N,E,S,W per piece index
    const uint32_t* cc;          // [ncolours][4][32] colour constraints
    uint32_t* infos;             // triangular stack: level L, info i at (S(S+1)-(S-L)(S-L+1))/2 + i, 32 words each
    GmState* state;
    uint32_t n, width, ncolours;
    unsigned long long push_budget;   // stop after this many pushes (0: none)
    unsigned long long placement_budget;  // stop once trials + pushes reach this (0: none)
    unsigned long long timeout_ns;    // stop after this long (0: none)
    GmGrid* grid = nullptr;           // multi-block search: the exchange area (zeroed before the launch)
};

size_t gm_smem_bytes();
cudaError_t launch_gm(const GmLaunch& P, cudaStream_t stream);
// The same search over `blocks` blocks of a cooperative launch (at most one per SM).
cudaError_t launch_gm_grid(const GmLaunch& P, uint32_t blocks, cudaStream_t stream);

}  // namespace emp
