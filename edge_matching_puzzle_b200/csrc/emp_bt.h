// Launch interface of the exhaustive backtracker kernels (emp_bt.cu).
#pragma once

#include "emp_layout.h"

#include <cuda_runtime.h>

#include <cstdint>

namespace emp {

// device status bits (BtLaunch::status)
enum : int {
    EMP_DEV_TIMEOUT = 1,    // the kernel passed its deadline and stopped
    EMP_DEV_ABORTED = 2,    // stopped early (deadline or cancel flag)
    EMP_DEV_SUPERSEDED = 8, // stop-at-first: subtrees after the first solution were cut
    EMP_DEV_FIRST_LOST = 16,// a wait for a first-solution record ran out (the record missed a solution)
};

// Lexicographically smallest solution path of a puzzle (its first solution in
// the reference's visiting order).
struct FirstRecord {
    unsigned int lock;
    unsigned int missed;    // a writer gave up waiting for the lock
    unsigned int has;
    unsigned int pad;
    uint16_t t[256];        // transition per level
};

// One solution found by a thread (solution dumps): its subtree, the placements of the
// subtree searched up to and including it (one thread searches the whole subtree in
// order), and its path.
struct SolutionRecord {
    unsigned long long orig;
    unsigned long long local;
    uint16_t t[256];
};

// Run state on the device, shared by the launches of one run.
struct BtRunCtl {
    unsigned long long deadline;     // absolute %globaltimer deadline of the run; 0 = none
    unsigned long long n_in;         // graph runs: records of the current round
    unsigned long long rounds;       // graph runs: DFS rounds launched
    unsigned long long records_in;   // graph runs: records read by all rounds
    unsigned long long records_out;  // graph runs: records handed back for a next round
    unsigned long long start_ns;     // %globaltimer at the start of the run
    unsigned long long first_found_ns;  // %globaltimer when the first solution was found (0: none)
    unsigned long long n_init;       // records of the run's first round (written by make_records)
};

struct BtLaunch {
    const uint32_t* tables = nullptr;         // all puzzle blobs
    const uint64_t* puzzle_offset = nullptr;  // word offset of each puzzle blob
    uint32_t depth = 0;                       // split depth (prefix expansion)
    uint32_t max_levels = 0;                  // max pieces over the puzzles of the launch
    uint32_t max_avail_words = 0;             // max 64-bit availability words (three kinds)
    uint32_t max_kw = 0;                      // max 64-bit candidate words of one kind
    uint64_t* spill = nullptr;                // [threads][max_levels][max_kw] remaining sets
    uint32_t smem_tab_words = 0;              // > 0: single puzzle, hot tables staged in shared memory
    // work records of this round and of the next one
    const uint32_t* in_rec = nullptr;
    uint64_t n_in = 0;
    uint32_t* out_rec = nullptr;
    unsigned long long* out_tail = nullptr;
    uint64_t out_capacity = 0;
    uint32_t rec_words = 0;                   // words per record
    uint32_t rec_r_off = 0;                   // offset of the remaining set in a record
    uint64_t item_budget = 0;                 // steps on a record before handing work back; 0 = never
    unsigned long long* cursor = nullptr;     // input queue head
    unsigned long long* totals = nullptr;     // per puzzle: [2p] nodes, [2p+1] solutions (subtrees only)
    unsigned long long* item_nodes = nullptr; // per initial subtree (optional)
    unsigned long long* item_sols = nullptr;
    unsigned long long* first_item = nullptr; // per puzzle: lowest initial subtree holding a solution
    FirstRecord* first_records = nullptr;     // per puzzle
    unsigned long long timeout_ns = 0;        // per-launch time limit (%globaltimer), 0: none
    int* abort_flag = nullptr;                // set by the host or by a stopping thread
    int* status = nullptr;
    int stop_at_first = 0;
    int stop_at_any = 0;                      // stop the whole run at the first solution found
    BtRunCtl* ctl = nullptr;                  // deadline; in graph runs also the round's record count
    int n_in_from_ctl = 0;                    // 1: read the round's record count from ctl->n_in
    uint32_t* incomplete = nullptr;           // per puzzle: 1 when some of its work was dropped (deadline, abort)
    SolutionRecord* sols = nullptr;           // solution dumps: every solution found (null: not recorded)
    unsigned long long* sol_count = nullptr;
    unsigned long long sol_capacity = 0;
    unsigned long long first_lock_wait_ns = 20000000ull;  // bound of a wait for a first-solution record
    uint32_t first_lock_init = 0;             // value the records' locks start at (1: held by nobody; tests)
    int stack_mode = kStackShared32;          // placement of the per-thread DFS stack (StackMode)
    uint32_t* stack = nullptr;                // kStackGlobal32: [blocks][max_levels][threads] stack entries
};

cudaError_t launch_expand(const BtLaunch& P, const uint16_t* parents, const uint32_t* parent_puzzle,
                          uint64_t n_parents, uint32_t level, uint32_t* counts, const uint64_t* offsets,
                          uint16_t* children, uint32_t* child_puzzle, unsigned long long* level_nodes,
                          unsigned long long* level_sols, int mode, cudaStream_t stream);
cudaError_t launch_scan(const uint32_t* counts, uint64_t n, uint64_t* offsets, uint64_t* block_sums,
                        uint64_t* grand_total, cudaStream_t stream);
uint64_t scan_block_sum_words(uint64_t n);
size_t dfs_smem_bytes(uint32_t max_levels, uint32_t max_avail_words, uint32_t threads, uint32_t tab_words,
                      int stack_mode);
uint32_t record_words(uint32_t max_levels, uint32_t max_kw);
cudaError_t launch_dfs(const BtLaunch& P, uint32_t blocks, uint32_t threads, cudaStream_t stream);
cudaError_t launch_bt_reset(const BtLaunch& P, uint32_t n_puzzles, cudaStream_t stream);
// frozen (per puzzle, may be null): puzzles whose prefixes are carried to the next
// level unchanged (a 0xFFFF pad), neither expanded nor counted
cudaError_t launch_expand_frozen(const BtLaunch& P, const uint16_t* parents, const uint32_t* parent_puzzle,
                                 uint64_t n_parents, uint32_t level, uint32_t* counts, const uint64_t* offsets,
                                 uint16_t* children, uint32_t* child_puzzle, unsigned long long* level_nodes,
                                 unsigned long long* level_sols, int mode, const uint8_t* frozen,
                                 cudaStream_t stream);
// puzzle_depth (per puzzle, may be null): prefix length of each puzzle's records;
// null = depth for all
// ctl (may be null): receives count in ctl->n_init, the first round's record count
cudaError_t launch_make_records(const uint16_t* prefixes, const uint32_t* prefix_puzzle, uint32_t depth,
                                uint64_t first, uint64_t stride, uint64_t count, uint32_t rec_words, uint32_t* rec,
                                cudaStream_t stream, const uint32_t* puzzle_depth = nullptr,
                                BtRunCtl* ctl = nullptr);
// Graph runs: the round controller (one thread) that turns this round's handed-back
// records into the next round's input and sets the loop condition, and the copy of
// those records into the input queue.
cudaError_t launch_round_advance(const BtLaunch& P, cudaGraphConditionalHandle loop, uint32_t max_rounds,
                                 cudaStream_t stream);
cudaError_t launch_round_copy(const BtLaunch& P, uint32_t* dst, const uint32_t* src, cudaStream_t stream);
// Solution dumps: for solution j, out[j] = placements of the sequential search up to
// and including it = (expansion nodes lexicographically at or before its prefix, one
// binary search per level array) + (counts of the subtrees before its own) + its local count.
cudaError_t launch_solution_index(const SolutionRecord* sols, uint64_t nsol, const uint16_t* const* level_prefixes,
                                  const uint64_t* level_counts, uint32_t depth, const unsigned long long* item_nodes,
                                  unsigned long long* out, cudaStream_t stream);
cudaError_t launch_record_prefix(const uint32_t* rec, uint32_t rec_words, uint64_t i, uint16_t* out,
                                 cudaStream_t stream);
const void* dfs_kernel_symbol(uint32_t max_kw, bool smem_tables, uint32_t threads, int stack_mode);

}  // namespace emp
