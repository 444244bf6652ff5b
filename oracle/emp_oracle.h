/*
 * CPU oracle for edge_matching_puzzle_b200 -- TEST INFRASTRUCTURE ONLY.
 *
 * This is a plain-C restatement of the reference's CPU search code, used as
 * the bit-exact checker of the CUDA kernels.  Only the test-suite, the smoke
 * check and the CPU-baseline leg of the benchmark may load it; the product
 * path (the CUDA library behind include/emp_b200.h) never calls it.
 *
 * What it restates (paths relative to the reference project root):
 *   - piece model: include/emp_piece.h:122-157 (kind, auto-similarity),
 *     :173-178 (rotation), :223-246 (binary piece encoding);
 *   - piece database: include/emp_piece_db.h:466-896 (kind indices, identical
 *     pieces and their masks, binary pieces), :1267-1312 (constraint table);
 *   - strategy orders: include/emp_basic_strategy_generator.h:44-53 (row
 *     major), include/emp_spiral_strategy_generator.h:52-100 (spiral);
 *   - exhaustive search: include/emp_strategy.h:159-265 (neighbour wiring),
 *     :332-415 (specific_run), include/emp_position_strategy.h:172-208;
 *   - solution dump: include/emp_situation_binary_dumper.h:58-124;
 *   - glutton max: include/CUDA_glutton_max.h:471-1637,
 *     include/CUDA_glutton_max_stack.h:271-522,
 *     include/CUDA_common_glutton.h:70-211.
 *
 * Parity pins: tests/golden holds the reference's own golden vectors
 * (tests/new_strategy_*, tests/CUDA_glutton_max_*, tests_CUDA/backtracker_*,
 * references/results.bin) and the oracle reproduces all of them.
 */
#ifndef EMP_ORACLE_H
#define EMP_ORACLE_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct op_puzzle op_puzzle;

/* colours: n*4 bytes, sides N,E,S,W of piece id (index+1); 0 = frame. */
op_puzzle *op_puzzle_create(uint32_t width, uint32_t height,
                            const uint8_t *colours, char *err, size_t err_len);
void op_puzzle_destroy(op_puzzle *p);

/* 1 when the puzzle contains identical pieces (the reference then needs its
 * HANDLE_IDENTICAL_PIECES build, emp_piece_db.h:885-896). */
int op_has_identical(const op_puzzle *p);
/* Number of pieces of a kind (0 centre, 1 border, 2 corner). */
uint32_t op_nb_kind(const op_puzzle *p, uint32_t kind);
/* Kind index of piece id-1 and the piece id of (kind, kind index). */
uint32_t op_kind_index(const op_puzzle *p, uint32_t piece_index);
uint32_t op_piece_of(const op_puzzle *p, uint32_t kind, uint32_t kind_index);
uint32_t op_border_color_id(const op_puzzle *p);
/* Orientation step of a piece: 1, 2 or 4 (2^auto_similarity). */
uint32_t op_orientation_step(const op_puzzle *p, uint32_t piece_index);
/* Identical-piece mask of (kind, transition t): nwords u64 written to out.
 * Returns the number of words of that kind's bitfield. */
uint32_t op_identical_mask(const op_puzzle *p, uint32_t kind, uint32_t t,
                           uint64_t *out, uint32_t max_words);
/* Constraint-table entry for a 4-slot code (emp_piece_db::get_pieces);
 * returns the bit size (0 when the code has no table entry). */
uint32_t op_table_entry(const op_puzzle *p, uint32_t code, uint64_t *out,
                        uint32_t max_words);
uint32_t op_color_id_size(const op_puzzle *p);

/* Position orders: fill order[n] with y*w+x in visiting order. */
void op_order_basic(uint32_t w, uint32_t h, uint32_t *order);
void op_order_spiral(uint32_t w, uint32_t h, uint32_t *order);

typedef struct {
    uint64_t nodes;              /* placements ("Total situations explored") */
    uint64_t solutions;          /* "Nb solutions" */
    uint64_t first_solution_nodes;
    uint32_t max_index;          /* deepest strategy index reached */
    int32_t status;              /* 0 complete, 1 node limit reached */
    uint16_t first_solution[256];/* per strategy index: transition t */
    uint32_t first_board[256];   /* per board position y*w+x: (id-1)<<2|o, 0xFFFFFFFF empty */
} op_bt_result;

/* Whole exhaustive search, exactly emp_strategy::specific_run.
 * results_bin: path to write the reference's results.bin (NULL: none).
 * maxlog: optional buffer receiving the "New max : k" / board lines. */
int op_bt_run(op_puzzle *p, const uint32_t *order, uint64_t node_limit,
              op_bt_result *out, const char *results_bin,
              char *maxlog, size_t maxlog_len);

/* The same search resumed from a partial situation, exactly
 * emp_strategy::set_initial_state (include/emp_strategy.h:418-467) followed by
 * specific_run: situation[l] is the transition placed at strategy level l for
 * l < placed (0 < placed < n).  Returns -2 when a transition of the situation is
 * not reachable in the reference's order, -1 on bad arguments. */
int op_bt_resume(op_puzzle *p, const uint32_t *order, const uint16_t *situation, uint32_t placed,
                 uint64_t node_limit, op_bt_result *out, const char *results_bin);

/* Prefix expansion to depth d: enumerate every placement path of levels
 * 0..d-1 in the reference's visiting order.  prefixes receives up to
 * max_prefixes*d transitions.  Returns the number of prefixes at depth d;
 * *nodes gets the placements at levels < d and *solutions the solutions
 * completed at levels < d. */
uint64_t op_bt_expand(op_puzzle *p, const uint32_t *order, uint32_t depth,
                      uint16_t *prefixes, uint64_t max_prefixes,
                      uint64_t *nodes, uint64_t *solutions);

/* Exhaustive count of the subtree below one prefix (levels >= d). */
int op_bt_subtree(op_puzzle *p, const uint32_t *order, const uint16_t *prefix,
                  uint32_t depth, uint64_t node_limit, uint64_t *nodes,
                  uint64_t *solutions);

/* Multi-threaded subtree counting over prefixes [begin,end) with nthreads
 * pthreads; per-prefix node/solution counts and the nodes per position kind
 * (kind_nodes[3], added to) are optional outputs. */
int op_bt_subtrees_parallel(op_puzzle *p, const uint32_t *order,
                            const uint16_t *prefixes, uint32_t depth,
                            uint64_t begin, uint64_t end, int nthreads,
                            uint64_t *nodes, uint64_t *solutions,
                            uint64_t *per_nodes, uint64_t *per_solutions,
                            uint64_t *kind_nodes);

/* Knuth random-probe estimate of the exhaustive tree size (sizing only). */
double op_bt_estimate(op_puzzle *p, const uint32_t *order, uint32_t probes,
                      uint64_t seed, double *per_level);

typedef struct {
    uint64_t placements;   /* trial evaluations + committed pushes */
    uint32_t max_level;    /* best number of pieces placed (m_max) */
    uint32_t level;        /* final stack level */
    int32_t status;        /* 0 full board, 1 budget reached, 2 exhausted */
    uint32_t played[256];      /* played info of the final stack */
    uint32_t max_played[256];  /* played info of the best partial board */
    uint64_t pushes, pops, levels_evaluated;
} op_gm_result;

/* Glutton max search (CUDA_glutton_max kernel semantics).  budget: stop after
 * that many placements (trials + pushes), push_budget: after that many
 * pushes, checked at the top of each level (0: none). */
int op_gm_run(op_puzzle *p, uint64_t budget, uint64_t push_budget, op_gm_result *out);
/* the glutton search's first situation: out[32 * pos + w], n positions */
int op_gm_initial(op_puzzle *p, uint32_t *out);

/* The reference's variable-space CUDA backtracker (feature CUDA_backtracker,
 * src/CUDA_backtracker.cu:67-178 with include/system_equation_for_CUDA.h:70-173 and
 * include/emp_variable_generator.h:335-621), row-major order, restated
 * sequentially.  Every selection is an event (elected lane, variable id
 * step<<10 | lane<<5 | bit, step): the kernel's "Thread L : selected variable V at
 * step S" lines.  solution_board[position] = (piece id-1)<<2 | orientation of the
 * first solution (0xFFFFFFFF when none).  max_selections > 0 stops after that many
 * selections.  Returns 0 when a solution was found, 1 otherwise, -1 on bad input. */
int op_vs_trace(op_puzzle *p, uint32_t max_events, uint32_t *ev_lane, uint32_t *ev_var, uint32_t *ev_step,
                uint32_t *n_events, uint32_t *solution_board, uint64_t max_selections);

#ifdef __cplusplus
}
#endif
#endif
