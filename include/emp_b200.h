/*
 * edge_matching_puzzle_b200 -- C ABI of the B200 search library.
 *
 * This is the boundary the reference's feature plugins call into.  In the
 * reference, feature_CUDA_backtracker::run (src/feature_CUDA_backtracker.cpp:
 * 31-38) calls
 *     void launch_CUDA_backtracker(const emp_piece_db&, const emp_FSM_info&,
 *                                  const emp_variable_generator&,
 *                                  const emp_strategy_generator&);
 * (include/feature_CUDA_backtracker.h:68-72) and feature_CUDA_glutton_max::run
 * (include/feature_CUDA_glutton_max.h:72-75) calls
 *     void launch_CUDA_glutton_max(const emp_piece_db&, const emp_FSM_info&);
 * (include/feature_CUDA_glutton_max.h:55-57).  Both launchers take the piece
 * database and the puzzle geometry; here those are flattened into
 * emp_puzzle_desc (piece colours + position order), and the results the
 * reference only prints are returned in plain structs.  The C++ launchers in
 * edge_matching_puzzle_b200/csrc/host keep the reference signatures and print
 * the reference's lines on top of this ABI.
 *
 * Rules: plain pointers and sizes only; no exception crosses the boundary;
 * every call returns an emp_status and emp_last_error() describes the last
 * failure of the calling thread.  A handle may be used by one call at a time.
 */
#ifndef EMP_B200_H
#define EMP_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EMP_ABI_VERSION 1u

typedef int32_t emp_status;
#define EMP_OK 0
#define EMP_INCOMPLETE 1          /* stopped by the timeout or a cancel: partial counts */
#define EMP_FIRST_LOST 2          /* counts complete and exact, but the first solution's board was not
                                     recorded: a thread's wait for the puzzle's first-solution record
                                     ran past first_lock_wait_us (has_first_solution is then 0) */
#define EMP_ERR_INVALID (-1)      /* bad argument or malformed puzzle */
#define EMP_ERR_UNSUPPORTED (-2)  /* valid input outside what the kernels support */
#define EMP_ERR_CUDA (-3)         /* CUDA runtime error (no device, launch failure...) */
#define EMP_ERR_NOMEM (-4)        /* device allocation failed */

/* Version of this ABI (EMP_ABI_VERSION). */
uint32_t emp_abi_version(void);

/* Message of the last failing call on this thread ("" when none). */
const char *emp_last_error(void);

/* Seeded puzzle generator of the project's workloads (splitmix64 stream):
 * frame-to-frame edges get colours 1..border_colors, other internal edges
 * border_colors+1..border_colors+interior_colors, outer edges 0; pieces are
 * shuffled and rotated.  colours_out receives 4*w*h bytes (N,E,S,W per piece).
 * Replaces the hand-written puzzle files of doc/example (no counterpart
 * function in the reference). */
emp_status emp_generate_puzzle(uint32_t width, uint32_t height, uint32_t border_colors,
                               uint32_t interior_colors, uint64_t seed, uint8_t *colours_out);

/* Puzzle description: what emp_pieces_parser::parse (include/emp_pieces_parser.h:
 * 53-101) and emp_strategy_generator (include/emp_strategy_generator.h:161-184)
 * provide to the reference's launchers. */
typedef struct emp_puzzle_desc {
    uint32_t width;
    uint32_t height;
    const uint8_t *colours;   /* 4*width*height bytes: N,E,S,W of piece id i+1; 0 = frame */
    const uint16_t *order;    /* width*height positions y*width+x in visiting order;
                                 NULL = row-major ("basic" strategy) */
} emp_puzzle_desc;

typedef struct emp_puzzle_t *emp_puzzle;

/* Builds the piece database (kinds, identical pieces, colour masks) and the
 * level plan of the order, as emp_piece_db's constructor (include/
 * emp_piece_db.h:466-1170) and emp_strategy's constructor (include/
 * emp_strategy.h:159-265) do.  Fails with EMP_ERR_INVALID on the inputs the
 * reference rejects (wrong kind counts, odd colour counts) and with
 * EMP_ERR_UNSUPPORTED beyond 256 pieces or colour id 30. */
emp_status emp_puzzle_create(const emp_puzzle_desc *desc, emp_puzzle *out);
void emp_puzzle_destroy(emp_puzzle puzzle);

typedef struct emp_puzzle_info {
    uint32_t width, height, nb_pieces;
    uint32_t nb_center, nb_border, nb_corner;
    uint32_t border_color_id;     /* max colour id + 1 (emp_piece_db.h:620) */
    uint32_t has_identical;       /* the reference needs HANDLE_IDENTICAL_PIECES */
    uint32_t identical_masks_with_extra;  /* transitions whose identical mask clears other candidates */
} emp_puzzle_info;

emp_status emp_puzzle_get_info(emp_puzzle puzzle, emp_puzzle_info *info);

/* Copies the puzzle's GPU table blob (header, per-side colour masks, level
 * plan, identical masks; layout in edge_matching_puzzle_b200/csrc/emp_model.h)
 * to out when capacity suffices; *words receives its size in 32-bit words.
 * Introspection for tests: no counterpart in the reference. */
emp_status emp_puzzle_export_tables(emp_puzzle puzzle, uint32_t *out, uint64_t capacity, uint64_t *words);

/* ---------------- exhaustive backtracker (emp_strategy semantics) ---------------- */

typedef struct emp_bt_config {
    uint32_t split_depth;        /* levels expanded before subtrees go to threads; 0 = auto */
    uint32_t threads_per_block;  /* 128, 256 or 512; 0 = the size with the most resident warps */
    uint32_t blocks_per_sm;      /* 0 = as many as fit */
    uint32_t stop_at_first;      /* 1: stop once the reference's first solution is known */
    uint64_t reserved_budget;    /* unused, keep 0 */
    uint32_t timeout_ms;         /* deadline of a whole run (all rounds), on the device clock; 0 = none */
    int32_t device;              /* CUDA device ordinal; -1 = current device */
    uint32_t keep_subtree_counts;/* 1: keep per-subtree counts for emp_bt_plan_subtree_counts */
    uint32_t split_budget;       /* once a round's queue is empty, a thread that spent this many
                                    DFS steps on its work record hands the rest back as new records
                                    for the next round; 0 = default (64 steps, or 2048 with
                                    a timeout_ms deadline) */
    uint32_t sample_stride;      /* emp_bt_count[_batch]: count only subtrees sample_first,
                                    sample_first+sample_stride, ...; 0 = all subtrees */
    uint32_t sample_first;
    uint32_t table_placement;    /* 0 = auto (shared memory for a single puzzle), 1 = global memory,
                                    2 = shared memory (single puzzle only) */
    uint32_t split_subtrees;     /* 0 = every puzzle is split at split_depth.  Otherwise each puzzle is
                                    split at its own depth: the first level at which it has at least
                                    this many subtrees, at most split_depth (0: no limit) and below
                                    its piece count.  For batches of puzzles of mixed sizes. */
    uint32_t use_graph;          /* 1: emp_bt_plan_run launches the whole run as one CUDA graph whose
                                    device-side loop (a conditional node) starts each next round;
                                    0: the host starts each round */
    uint32_t stop_at_any;        /* 1: stop the whole run at the first solution found by any thread
                                    (time to a first solution; counts are then partial) */
    uint32_t first_lock_wait_us; /* bound of a thread's wait for its puzzle's first-solution record,
                                    which another thread holds for a few hundred cycles; 0 = 20000.
                                    A wait that runs out reports EMP_FIRST_LOST for the puzzle */
    uint32_t hold_first_lock;    /* testing only: 1 = every first-solution record starts locked by
                                    nobody, so each wait runs out (exercises EMP_FIRST_LOST) */
    uint32_t stack_placement;    /* where each thread keeps its DFS stack: 0 = default (1 when
                                    the tables are staged in shared memory and 1 leaves at
                                    least 16 warps per SM, else 3),
                                    1 = shared memory, 32-bit entries with the placed piece's colours,
                                    2 = shared memory, 16-bit entries (more threads per SM; colours are
                                        read from the transition table),
                                    3 = global memory (L1-cached), 32-bit entries,
                                    4 = one DFS per warp: the warp's stack in shared memory,
                                        lane w evaluates candidate word w and a ballot picks
                                        the next candidate (kinds up to 32 words; 1 to 3
                                        take 16) */
} emp_bt_config;

typedef struct emp_bt_result {
    uint64_t solutions;          /* "Nb solutions" (include/emp_strategy.h:413) */
    uint64_t nodes;              /* "Total situations explored" (:412) */
    uint64_t subtrees;           /* prefixes at the split depth */
    uint64_t expansion_nodes;    /* placements at levels below the split depth */
    int32_t status;              /* EMP_OK, or EMP_INCOMPLETE when part of this puzzle's search was
                                    dropped (deadline or cancel): its counts are then partial */
    uint32_t split_depth;        /* this puzzle's split depth */
    uint32_t has_first_solution;
    uint32_t first_solution[256];/* per board position y*w+x: (piece id-1)<<2 | orientation */
    double kernel_ms;            /* DFS kernel time (device events, all rounds) */
    double total_ms;             /* whole call, host clock */
    uint32_t rounds;             /* DFS rounds (work handed back between rounds) */
    uint32_t first_found_us;     /* device time from the start of the run to the first solution
                                    found by any thread, in microseconds; 0 = none found */
    double dfs_busy_ms;          /* sum of the DFS launches' device times (no gaps between rounds) */
    uint64_t work_records;       /* work records read by the DFS launches (all rounds) */
    uint64_t handed_back;        /* work records written back for a next round */
} emp_bt_result;

/* Exhaustive count of one puzzle: every solution and every placement of the
 * reference's search (position 0 keeps its first candidate, emp_strategy.h:389).
 * With config->sample_stride set, only the sampled subtrees are counted and
 * nodes/solutions hold their counts (expansion_nodes still reports the levels
 * below the split depth). */
emp_status emp_bt_count(emp_puzzle puzzle, const emp_bt_config *config, emp_bt_result *result);

/* The same search resumed from a partial situation, as the reference's
 * --initial_situation parameter does for new_strategy: emp_strategy::set_initial_state
 * followed by specific_run (include/emp_strategy.h:418-467, 343-410).  situation[l] is
 * the transition t = kind_index<<2 | orientation placed at level l of the puzzle's
 * order, for l < placed (the situation string's pieces up to its first empty position
 * in that order).  As in the reference, the search restarts the last placed level
 * from its first candidate, continues with the candidates every shallower level has
 * left after the situation's piece, and ends when level 1 is exhausted; nodes and
 * solutions count that search alone.  placed <= 1 is a whole search (emp_bt_count).
 * A situation piece that the reference's order cannot reach is EMP_ERR_INVALID. */
emp_status emp_bt_resume(emp_puzzle puzzle, const uint16_t *situation, uint32_t placed,
                         const emp_bt_config *config, emp_bt_result *result);

/* Same for many puzzles in one persistent launch; results[i] per puzzle. */
emp_status emp_bt_count_batch(const emp_puzzle *puzzles, uint32_t count, const emp_bt_config *config,
                              emp_bt_result *results);

/* One solution of the exhaustive search, placed where the reference's sequential
 * search finds it. */
typedef struct emp_bt_solution {
    uint64_t node_index;         /* placements made by the sequential search up to and including this
                                    solution: the count the reference's results.bin stores with it
                                    (include/emp_situation_binary_dumper.h:103-117) */
    uint32_t board[256];         /* per board position y*w+x: (piece id-1)<<2 | orientation */
} emp_bt_solution;

/* Every solution of one puzzle in the reference's order, with its node index: what
 * emp_strategy writes to results.bin (include/emp_strategy.h:367-375).  The search runs
 * without handing work between threads (each subtree is searched in order by one
 * thread), so it is slower than emp_bt_count on large trees.  *found receives the
 * number of solutions; out receives the first min(found, capacity) of them in the
 * reference's order (when found > capacity the search runs a second time keeping all
 * of them, at most 2^20, to rank them; more than that fails with EMP_ERR_UNSUPPORTED). */
emp_status emp_bt_solutions(emp_puzzle puzzle, const emp_bt_config *config, emp_bt_solution *out, uint64_t capacity,
                            uint64_t *found, emp_bt_result *result);

/* emp_bt_solutions of the search resumed from a partial situation (emp_bt_resume):
 * what the reference's new_strategy with --initial_situation writes to results.bin,
 * each solution with the placements of the resumed search up to it. */
emp_status emp_bt_resume_solutions(emp_puzzle puzzle, const uint16_t *situation, uint32_t placed,
                                   const emp_bt_config *config, emp_bt_solution *out, uint64_t capacity,
                                   uint64_t *found, emp_bt_result *result);

/* Debug mode: the reference's own CUDA_backtracker search, the variable-space
 * single-warp backtracker of src/CUDA_backtracker.cu:67-178 (variables and
 * transition vectors of include/emp_variable_generator.h:335-621 and
 * include/system_equation_for_CUDA.h:70-173), row-major puzzles of at most 64
 * pieces.  Each selection is an event, the kernel's "Thread L : selected variable
 * V at step S" line; *found = 1 and board[position] = (piece id-1)<<2 |
 * orientation when it reached a solution (the reference's first solution, which
 * the exhaustive search's first_solution also gives).  max_selections > 0 and
 * timeout_ms (0 = 60 s) bound the run (EMP_INCOMPLETE). */
typedef struct emp_vs_event {
    uint32_t lane;               /* the elected lane */
    uint32_t variable;           /* step << 10 | lane << 5 | bit */
    uint32_t step;
} emp_vs_event;

emp_status emp_bt_variable_space(emp_puzzle puzzle, int device, uint64_t max_selections, uint32_t timeout_ms,
                                 emp_vs_event *events, uint64_t capacity, uint64_t *n_events, uint32_t *board,
                                 uint32_t *found);

/* Split form of the batch call: plan (upload + prefix expansion), run (kernel
 * launch on a stream, asynchronous), results (synchronise + download). */
typedef struct emp_bt_plan_t *emp_bt_plan;

emp_status emp_bt_plan_create(const emp_puzzle *puzzles, uint32_t count, const emp_bt_config *config,
                              emp_bt_plan *out);
/* Number of subtrees of the plan (all puzzles). */
emp_status emp_bt_plan_subtrees(emp_bt_plan plan, uint64_t *subtrees);
/* Restrict the next runs to subtrees first, first+stride, ... (count of them). */
emp_status emp_bt_plan_select(emp_bt_plan plan, uint64_t first, uint64_t stride, uint64_t count);
/* Launch on stream (a cudaStream_t; NULL = default stream). */
emp_status emp_bt_plan_run(emp_bt_plan plan, void *stream);
/* Wait for the last run and fill results[count] (per puzzle). */
emp_status emp_bt_plan_results(emp_bt_plan plan, emp_bt_result *results);
/* Per-subtree counts of the last run in selection order (needs keep_subtree_counts). */
emp_status emp_bt_plan_subtree_counts(emp_bt_plan plan, uint64_t *nodes, uint64_t *solutions,
                                      uint64_t capacity);
/* Prefix (split_depth transitions t = kind_index<<2|orientation) of a selected subtree. */
emp_status emp_bt_plan_subtree_prefix(emp_bt_plan plan, uint64_t index, uint16_t *prefix, uint32_t capacity);
void emp_bt_plan_destroy(emp_bt_plan plan);

/* ---------------- autotuner (no counterpart in the reference) ---------------- */

typedef struct emp_bt_tune_result {
    emp_bt_config best;          /* base configuration with the tuned fields of the fastest trial */
    double best_rate;            /* its placements per second of device time */
    double default_rate;         /* the first trial's rate (base configuration, library defaults) */
    uint32_t trials;             /* configurations timed */
    uint32_t reserved;
} emp_bt_tune_result;

/* Chooses the launch parameters for a set of puzzles by timing short runs on the
 * device.  Starting from base (NULL = defaults), it tunes one field at a time, keeping
 * each field's fastest value before moving on:
 *   stack_placement     the DFS stack in shared memory (32- or 16-bit entries) or global memory,
 *                       or one DFS per warp (tried first when the kinds are too wide for the others)
 *   threads_per_block   128, 256, 512
 *   split_subtrees      per-puzzle split targets (batches of several puzzles) or
 *   split_depth         split depths (a single puzzle)
 *   split_budget        steps before a thread hands work back
 *   table_placement     shared or global memory (a single puzzle)
 * Every trial builds a plan (upload and prefix expansion, not timed) and runs it with
 * a deadline of trial_ms; its rate is the placements counted divided by the run's
 * device time. */
emp_status emp_bt_autotune(const emp_puzzle *puzzles, uint32_t count, const emp_bt_config *base,
                           uint32_t trial_ms, emp_bt_tune_result *out);

/* ---------------- learned value ordering (no counterpart in the reference) ----------------
 *
 * A network scores candidate placements (position, piece, rotation) from 512
 * features of the placement and the pieces already placed: one-hot side colours,
 * neighbour states, how many edges of each free side's colour remain on unplaced
 * pieces, position, depth and kind.  It has two hidden layers of 256 (relu) and one
 * output s; sigmoid(s) reads as the chance that the placement lies on a solution
 * path.  Inference runs on the tensor cores (BF16 operands, FP32 accumulation),
 * training in f32 CUDA kernels.  Ordering changes only which subtrees are searched
 * first: the set of subtrees and the search below them are those of the plain
 * order, so exhaustive counts do not change. */

#define EMP_MLP_INPUTS 512u
#define EMP_MLP_HIDDEN 256u
/* parameters in this order: W1[256][512], b1[256], W2[256][256], b2[256], w3[256], b3 */
#define EMP_MLP_PARAMS (256u * 512u + 256u + 256u * 256u + 256u + 256u + 1u)

typedef struct emp_mlp_t *emp_mlp;

/* A network with seeded random weights (uniform, scaled by 1/sqrt(fan-in)) on a device. */
emp_status emp_mlp_create(uint64_t seed, int32_t device, emp_mlp *out);
void emp_mlp_destroy(emp_mlp model);
emp_status emp_mlp_get_params(emp_mlp model, float *params);        /* EMP_MLP_PARAMS values */
emp_status emp_mlp_set_params(emp_mlp model, const float *params);

/* Feature rows of n candidates: candidate cands[i] placed at level lens[i] after the
 * transitions prefixes[i*stride .. i*stride+lens[i]) of the puzzle's order.  out
 * receives n * EMP_MLP_INPUTS values (0 or 1). */
emp_status emp_mlp_features(emp_puzzle puzzle, const uint16_t *prefixes, uint32_t stride, const uint16_t *lens,
                            const uint16_t *cands, uint64_t n, float *out);

/* Scores of n feature rows on the tensor cores (features rounded to BF16). */
emp_status emp_mlp_score(emp_mlp model, const float *features, uint64_t n, float *scores);
/* Same network in f32 on the CUDA cores (the training forward pass). */
emp_status emp_mlp_score_f32(emp_mlp model, const float *features, uint64_t n, float *scores);

/* Weighted logistic loss of n rows with labels in {0,1}: loss = sum w (softplus(s) - y s) / sum w,
 * and its gradient with respect to every parameter (EMP_MLP_PARAMS values). */
emp_status emp_mlp_loss_grad(emp_mlp model, const float *features, const float *labels, const float *weights,
                             uint64_t n, double *loss, float *grads);

typedef struct emp_mlp_train_config {
    uint32_t epochs;             /* passes over the samples; 0 = 30 */
    uint32_t batch;              /* rows per step; 0 = 2048 */
    float learning_rate;         /* Adam step size; 0 = 1e-3 */
    uint32_t seed;               /* shuffling */
    uint32_t max_level;          /* train on levels below this one only (the levels an ordered plan
                                    scores: its split depth); 0 = every level */
    uint32_t reserved[3];
} emp_mlp_train_config;

typedef struct emp_mlp_train_report {
    uint64_t samples;            /* candidate placements seen by training */
    uint64_t positives;          /* of them on the solution paths */
    uint32_t puzzles;            /* puzzles with a solution path */
    uint32_t epochs;
    double first_loss;           /* mean weighted loss of the first and the last epoch */
    double last_loss;
    double train_ms;
} emp_mlp_train_report;

/* Trains the network on the solver's traces: for every puzzle with a solution
 * (solutions[i*256 ..] in the emp_bt_result.first_solution format, 0xFFFFFFFF for
 * none), every level of the solution path gives one positive (the solution's
 * placement) and its siblings (the other candidates the search tries at that node)
 * as negatives; positives are weighted to balance the two classes. */
emp_status emp_mlp_train(emp_mlp model, const emp_puzzle *puzzles, uint32_t count, const uint32_t *solutions,
                         const emp_mlp_train_config *config, emp_mlp_train_report *report);

/* Queues the plan's subtrees best first: every prefix gets the sum over its levels of
 * log sigmoid(score of the placement), and within each puzzle the subtrees run in
 * decreasing order of that sum.  Counts stay those of the plain order; stop_at_first
 * (the lexicographically first solution) is not available on an ordered plan. */
emp_status emp_bt_plan_order(emp_bt_plan plan, emp_mlp model);

/* ---------------- glutton max search (CUDA_glutton_max semantics) ---------------- */

typedef struct emp_gm_config {
    uint64_t push_budget;        /* stop after this many committed placements; 0 = none */
    uint32_t timeout_ms;         /* stop after this long on the device; 0 = one hour */
    int32_t device;              /* CUDA device ordinal; -1 = current device */
    uint64_t placement_budget;   /* stop at the first level that starts with at least this many
                                    placements done (candidate trial evaluations + committed
                                    placements, the kernel's own count); 0 = none */
    uint32_t blocks;             /* blocks of the search, at most one per SM: every block keeps a copy
                                    of the level and the trials of each validity pass are shared out
                                    over all of them; 0 = one per SM, 1 = a single block */
    uint32_t reserved[5];
} emp_gm_config;

typedef struct emp_gm_result {
    int32_t status;              /* 0 full board, 1 stopped by budget or timeout, 2 search exhausted
                                    (the reference's "Empty stack") */
    uint32_t max_level;          /* most pieces placed at once (the stack's m_max) */
    uint32_t level;              /* pieces placed in the final stack */
    uint32_t reserved0;
    uint32_t best_board[256];    /* best partial board: per position y*w+x (piece id-1)<<2 | orientation,
                                    0xFFFFFFFF empty */
    uint32_t final_board[256];   /* final stack (the reference's "Situation with stack played info") */
    uint64_t trials;             /* candidate trial evaluations (all validity passes) */
    uint64_t pushes;             /* committed placements */
    uint64_t pops;
    uint64_t passes;             /* validity passes */
    uint64_t levels;             /* levels evaluated */
    double kernel_ms;
} emp_gm_result;

/* Greedy max-placement search of one puzzle, as launch_CUDA_glutton_max
 * (src/CUDA_glutton_max.cu:38-108) runs it: the same level-by-level choice of
 * the best candidate, the same backtracking, the same final board. */
emp_status emp_glutton_max(emp_puzzle puzzle, const emp_gm_config *config, emp_gm_result *result);

/* The same search as emp_glutton_max, with the same results, but it allocates
 * no device memory. This entry point has no counterpart in the reference.
 *
 * It is for callers that must not allocate once they are running. One example
 * is a service that sizes its device memory at start-up and must not hit an
 * out-of-memory error halfway through a job. Another is a loop that shares
 * the GPU with other streams: cudaFree synchronises the whole device and
 * would stall them.
 *
 * Its device memory is one array of 4,232,448 bytes compiled into this
 * library, one copy per device. That is enough for every puzzle the library
 * accepts: up to 256 pieces and colour ids up to 30 (emp_puzzle_create refuses
 * higher ids). Larger puzzles are rejected with EMP_ERR_UNSUPPORTED and a
 * message naming the limit.
 *
 * The search runs on one block of one SM: config->blocks is ignored (the
 * multi-block search of emp_glutton_max keeps its exchange buffers in
 * allocated memory).
 *
 * Every call looks up the array's device address on the current device (this
 * allocates nothing); the first call on a device also loads the array onto
 * it. Make that first call before any stream capture begins.
 *
 * Every call shares the array, and the array keeps whatever the previous call
 * left. Each call rewrites everything the search reads before writing it.
 * Calls that overlap on the same device, from several host threads, race on
 * the array: the caller must serialise them.
 *
 * kernel_ms is the host's wall time from the launch to the return of the result. */
emp_status emp_glutton_max_noalloc(emp_puzzle puzzle, const emp_gm_config *config, emp_gm_result *result);

/* ---------------- glutton wide (feature_CUDA_glutton_wide, include/feature_CUDA_glutton_wide.h) ----------------
 * The reference's CUDA glutton wide prepares its first situation and prints it
 * (src/CUDA_glutton_wide.cu:27-37; the search itself is not written there).  That
 * situation is the level the glutton max search starts from: every position's info,
 * with corner and border pieces in their forced orientation and centre pieces in all
 * four (include/CUDA_common_glutton.h:150-211).  infos[32 * j + w] receives word w of
 * position j's info, bit 4 * (piece % 8) + orientation of word piece / 8 (piece ids
 * from 0), for the width * height positions; at level 0 info index j is position j.
 * capacity_words must be at least 32 * width * height. */
emp_status emp_glutton_wide_situation(emp_puzzle puzzle, uint32_t *infos, uint64_t capacity_words);

#ifdef __cplusplus
}
#endif
#endif /* EMP_B200_H */
