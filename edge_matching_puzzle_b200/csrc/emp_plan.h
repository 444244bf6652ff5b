// Exhaustive backtracker plan (the state behind emp_bt_plan): shared by the
// plan's C ABI (emp_api.cu) and the learned ordering (emp_learn_api.cu).
#pragma once

#include "emp_b200.h"
#include "emp_bt.h"
#include "emp_common.h"

#include <cuda_runtime.h>

#include <vector>

using emp::DeviceBuffer;

struct emp_bt_plan_t {
    std::vector<emp_puzzle> puzzles;
    emp_bt_config cfg{};
    int device = 0;
    uint32_t depth = 0, max_levels = 0, max_avail = 0, max_kw = 0;
    uint32_t threads = 128, blocks = 0, rec_words = 0, smem_tab_words = 0;
    uint64_t capacity = 0, budget = 0;
    DeviceBuffer tables, poff;
    DeviceBuffer prefixes, prefix_puzzle;     // split-depth prefixes (all)
    DeviceBuffer rec_init, rec_a, rec_b;      // initial records (selection), round queues
    DeviceBuffer counters;                    // [0] cursor, [1] output tail
    DeviceBuffer totals, first_item, records, flags, item_nodes, item_sols, spill, prefix_out;
    DeviceBuffer stack;                       // kStackGlobal32: the threads' DFS stacks
    int stack_mode = emp::kStackShared32;
    DeviceBuffer ctl, incomplete, puzzle_depth_dev;
    std::vector<uint32_t> puzzle_depth;       // per puzzle split depth
    bool adaptive = false;                    // per puzzle split depths (split_subtrees)
    cudaStream_t capture_stream = nullptr;    // graph runs: stream the graph is captured on
    cudaStream_t select_stream = nullptr;     // initial records of a selection are built here ...
    cudaEvent_t ev_select = nullptr;          // ... and a run waits for this event before it starts
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    const void* graph_rec_init = nullptr;     // the initial-record buffer the graph was captured with
    bool graph_ran = false;
    // solution dumps: the expansion's level arrays (prefixes of length L at [L]) and
    // the solutions found
    bool dump = false;
    std::vector<DeviceBuffer> level_prefixes;
    std::vector<uint64_t> level_counts;
    DeviceBuffer sol_buf, sol_count;
    uint64_t sol_capacity = 0;
    uint64_t n_all = 0, n_init = 0;
    bool sampled = false;
    bool resumed = false;                     // initial records of a resumed search (emp_bt_resume)
    std::vector<unsigned long long> exp_nodes, exp_sols;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, evr0 = nullptr, evr1 = nullptr;
    bool ran = false;
    uint32_t rounds = 0;
    double busy_ms = 0;
    uint64_t records_in = 0, records_out = 0;

    void drop_graph()
    {
        if (graph_exec) cudaGraphExecDestroy(graph_exec);
        if (graph) cudaGraphDestroy(graph);
        graph_exec = nullptr;
        graph = nullptr;
        graph_rec_init = nullptr;
    }

    ~emp_bt_plan_t()
    {
        drop_graph();
        if (capture_stream) cudaStreamDestroy(capture_stream);
        if (select_stream) cudaStreamDestroy(select_stream);
        if (ev_select) cudaEventDestroy(ev_select);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (evr0) cudaEventDestroy(evr0);
        if (evr1) cudaEventDestroy(evr1);
    }

    emp::BtLaunch launch() const
    {
        emp::BtLaunch P;
        P.tables = tables.as<uint32_t>();
        P.puzzle_offset = poff.as<uint64_t>();
        P.depth = depth;
        P.max_levels = max_levels;
        P.max_avail_words = max_avail;
        P.max_kw = max_kw;
        P.spill = spill.as<uint64_t>();
        P.smem_tab_words = smem_tab_words;
        P.rec_words = rec_words;
        P.rec_r_off = rec_words - 2 * max_kw;
        P.out_capacity = capacity;
        P.item_budget = budget;
        unsigned long long* c = counters.as<unsigned long long>();
        P.cursor = c;
        P.out_tail = c + 1;
        P.totals = totals.as<unsigned long long>();
        P.item_nodes = item_nodes.as<unsigned long long>();
        P.item_sols = item_sols.as<unsigned long long>();
        P.first_item = first_item.as<unsigned long long>();
        P.first_records = records.as<emp::FirstRecord>();
        P.timeout_ns = static_cast<unsigned long long>(cfg.timeout_ms) * 1000000ull;
        P.abort_flag = flags.as<int>();
        P.status = flags.as<int>() + 1;
        P.stop_at_first = cfg.stop_at_first ? 1 : 0;
        P.stop_at_any = cfg.stop_at_any ? 1 : 0;
        P.ctl = ctl.as<emp::BtRunCtl>();
        P.sols = sol_buf.as<emp::SolutionRecord>();
        P.sol_count = sol_count.as<unsigned long long>();
        P.sol_capacity = sol_capacity;
        P.incomplete = incomplete.as<uint32_t>();
        if (cfg.first_lock_wait_us) P.first_lock_wait_ns = 1000ull * cfg.first_lock_wait_us;
        P.first_lock_init = cfg.hold_first_lock ? 1u : 0u;
        P.stack_mode = stack_mode;
        P.stack = stack.as<uint32_t>();
        return P;
    }
};

// Initial work records for subtrees first, first+stride, ... (count of them), in the
// order of the plan's prefix array.
emp_status plan_build_initial(emp_bt_plan_t& pl, uint64_t first, uint64_t stride, uint64_t count);
