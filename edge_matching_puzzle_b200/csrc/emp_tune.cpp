// Autotuner of the exhaustive backtracker's launch parameters (emp_bt_autotune).
//
// Coordinate descent over timed trial runs: each trial is a plan built with one
// candidate configuration and run under a deadline; the rate compared is the
// placements counted per second of device time of the run.
#include "emp_b200.h"
#include "emp_common.h"

#include <algorithm>
#include <string>
#include <vector>

using emp::fail;

namespace {

struct Trial {
    const emp_puzzle* puzzles;
    uint32_t count;
    uint32_t trial_ms;
    uint32_t runs = 0;
};

// placements/s of one configuration; negative when the configuration cannot run
// (for example a block size whose per-thread state does not fit shared memory)
double time_config(Trial& t, const emp_bt_config& cfg)
{
    emp_bt_config c = cfg;
    c.timeout_ms = t.trial_ms;
    c.sample_stride = 0;
    c.keep_subtree_counts = 0;
    emp_bt_plan plan = nullptr;
    if (emp_bt_plan_create(t.puzzles, t.count, &c, &plan) != EMP_OK) return -1.0;
    std::vector<emp_bt_result> res(t.count);
    double rate = -1.0;
    if (emp_bt_plan_run(plan, nullptr) == EMP_OK && emp_bt_plan_results(plan, res.data()) == EMP_OK) {
        uint64_t nodes = 0;
        for (const emp_bt_result& r : res) nodes += r.nodes - r.expansion_nodes;
        const double ms = res[0].kernel_ms;
        rate = ms > 0 ? nodes / (ms / 1000.0) : 0.0;
    }
    emp_bt_plan_destroy(plan);
    ++t.runs;
    return rate;
}

}  // namespace

extern "C" emp_status emp_bt_autotune(const emp_puzzle* puzzles, uint32_t count, const emp_bt_config* base,
                                      uint32_t trial_ms, emp_bt_tune_result* out)
{
    emp::clear_error();
    if (!puzzles || !count || !out) return fail(EMP_ERR_INVALID, "emp_bt_autotune: no puzzle");
    if (!trial_ms) return fail(EMP_ERR_INVALID, "emp_bt_autotune: trial_ms must be positive");
    emp_bt_config best{};
    best.device = -1;
    if (base) best = *base;
    best.stop_at_first = 0;
    Trial t{puzzles, count, trial_ms};
    double best_rate = time_config(t, best);
    if (best_rate < 0 && !best.stack_placement) {
        best.stack_placement = 4;  // kinds wider than the per-thread search takes: one DFS per warp
        best_rate = time_config(t, best);
        if (best_rate < 0) best.stack_placement = 0;
    }
    if (best_rate < 0)
        return fail(EMP_ERR_INVALID, "emp_bt_autotune: the base configuration does not run: " + emp::last_error());
    const double default_rate = best_rate;
    auto consider = [&](const emp_bt_config& cand) {
        const double r = time_config(t, cand);
        if (r > best_rate) {
            best_rate = r;
            best = cand;
        }
    };
    // the DFS stack: shared 32-bit, shared 16-bit, global, one per warp
    for (uint32_t placement : {1u, 2u, 3u, 4u}) {
        if (placement == best.stack_placement) continue;  // 0, the default, is none of them
        emp_bt_config c = best;
        c.stack_placement = placement;
        consider(c);
    }
    for (uint32_t threads : {128u, 256u, 512u}) {
        if (threads == best.threads_per_block) continue;
        emp_bt_config c = best;
        c.threads_per_block = threads;
        consider(c);
    }
    if (count > 1) {
        for (uint32_t target : {256u, 1024u, 4096u, 16384u}) {
            if (target == best.split_subtrees) continue;
            emp_bt_config c = best;
            c.split_subtrees = target;
            consider(c);
        }
    } else {
        for (uint32_t depth : {8u, 10u, 12u, 14u, 16u}) {
            if (depth == best.split_depth) continue;
            emp_bt_config c = best;
            c.split_depth = depth;
            consider(c);
        }
    }
    for (uint32_t budget : {64u, 256u, 512u, 2048u, 8192u}) {
        if (budget == best.split_budget) continue;
        emp_bt_config c = best;
        c.split_budget = budget;
        consider(c);
    }
    if (count == 1) {
        for (uint32_t placement : {1u, 2u}) {
            if (placement == best.table_placement) continue;
            emp_bt_config c = best;
            c.table_placement = placement;
            consider(c);
        }
    }
    emp::clear_error();  // failed candidates are skipped, not reported
    out->best = best;
    out->best.timeout_ms = base ? base->timeout_ms : 0;
    out->best_rate = best_rate;
    out->default_rate = default_rate;
    out->trials = t.runs;
    out->reserved = 0;
    return EMP_OK;
}
