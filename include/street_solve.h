/*
 * street_solve.h -- C ABI of the B200 single-street N-player Linear-CFR
 * subgame solver.
 *
 * Drop-in for the reference interface src/cuda/street_solve.cuh: the structs
 * SSNode / SSTreeData / SSOutput keep the reference field order, types and
 * sizes byte for byte (street_solve.cuh:52-65, 69-122, 126-143), and the four
 * entry points keep the reference names, argument meaning and "0 on success"
 * convention (street_solve.cuh:172-194), so python/street_solver_gpu.py and
 * python/leaf_values.py bind this library unchanged.
 *
 * Two builds of the same source differ only in SS_MAX_HANDS, which is part
 * of the SSTreeData layout:
 *   libstreet_solve.so       SS_MAX_HANDS = 200   (reference layout)
 *   libstreet_solve_wide.so  SS_MAX_HANDS = 1326  (every 2-card combo)
 * ss_abi_info() reports which one is loaded.
 *
 * Entry points marked EXTENSION have no counterpart in the reference.
 */
#ifndef B200_STREET_SOLVE_H
#define B200_STREET_SOLVE_H

#include <stdint.h>

/* ── Limits (street_solve.cuh:35-42) ─────────────────────────────────── */

#define SS_MAX_PLAYERS     6
#ifndef SS_MAX_HANDS
#define SS_MAX_HANDS       200
#endif
#define SS_MAX_ACTIONS     8
#define SS_MAX_TREE_NODES  4096   /* informational, as in the reference (never enforced there) */
#define SS_MAX_BOARD       5
#define SS_MAX_LEAVES      64     /* informational, as in the reference */
#define SS_NUM_CONT_STRATS 4
#define SS_MAX_RAISES      3      /* default raise cap of ss_build_tree */

/* Node types (street_solve.cuh:45-49) */
#define SS_NODE_DECISION  0
#define SS_NODE_FOLD      1
#define SS_NODE_SHOWDOWN  2
#define SS_NODE_LEAF      4

/* Return codes.  0 is success; every failure is negative, so callers that
 * test "!= 0" (the reference convention, street_solve.cu:29-36) still work. */
#define SS_OK                0
#define SS_ERR_INVALID      -1   /* malformed tree, ranges or arguments */
#define SS_ERR_CUDA         -2   /* CUDA runtime or launch failure */
#define SS_ERR_NOMEM        -3   /* device or host allocation failed */
#define SS_ERR_UNSUPPORTED  -4   /* terminal class this build cannot solve at this size */
#define SS_ERR_NO_DEVICE    -5   /* no CUDA device */

/* ── Flat tree node (street_solve.cuh:52-65), 26 x int32 = 104 bytes ─── */

typedef struct {
    int type;                     /* SS_NODE_* */
    int player;                   /* acting player at decisions; winner at folds; -1 otherwise */
    int num_children;
    int first_child;              /* index into SSTreeData.children */
    int pot;                      /* chips */
    int bets[SS_MAX_PLAYERS];     /* each player's total bet this street */
    int board_cards[5];
    int num_board;
    int leaf_idx;                 /* SS_NODE_LEAF: row of leaf_values */
    int fold_player;              /* kept for layout; the builder leaves it -1 */
    int num_players;              /* active (non-folded) players at this node */
    int active_players[SS_MAX_PLAYERS];
} SSNode;

/* ── Solver input (street_solve.cuh:69-122) ──────────────────────────── */

typedef struct {
    SSNode *nodes;
    int *children;
    int num_nodes;
    int num_children_total;

    int num_players;

    int hands[SS_MAX_PLAYERS][SS_MAX_HANDS][2];
    float weights[SS_MAX_PLAYERS][SS_MAX_HANDS];
    int num_hands[SS_MAX_PLAYERS];

    int board[SS_MAX_BOARD];
    int num_board;

    /* leaf_values[leaf_idx * num_players * max_hands + p * max_hands + h],
     * max_hands = max(num_hands).  Caller-owned: ss_free_tree never frees it. */
    float *leaf_values;
    int num_leaves;

    int *level_order;
    int *node_depth;
    int max_depth;

    int *decision_node_indices;
    int num_decision_nodes;
    int *showdown_node_indices;
    int num_showdown_nodes;
    int *leaf_node_indices;
    int num_leaf_nodes;
    int *fold_node_indices;
    int num_fold_nodes;

    int starting_pot;
    int effective_stack;
    int is_river;

    /* frozen_action[node] = action index forced at that node for every hand
     * (-1 = free); NULL disables freezing.  Caller-owned. */
    int *frozen_action;
} SSTreeData;

/* ── Solver output (street_solve.cuh:126-143) ────────────────────────── */

typedef struct {
    float *root_strategy;         /* [root_num_actions][num_hands[root_player]], last iterate */
    int root_num_actions;
    int root_player;
    float *root_ev;               /* [num_players][max_hands]; row 0 = root values of the last traverser */
    float *avg_strategies;        /* [num_avg_nodes][SS_MAX_ACTIONS][max_hands] */
    int *avg_strategy_node_ids;   /* [num_avg_nodes], decision nodes in index order */
    int num_avg_nodes;
    int num_players;
    int max_hands;
} SSOutput;

/* ── EXTENSION types ─────────────────────────────────────────────────── */

typedef struct {
    int abi_version;              /* 1 */
    int max_hands;                /* SS_MAX_HANDS of this build */
    int max_players;
    int max_actions;
    int sizeof_node;
    int sizeof_tree;
    int sizeof_output;
} SSAbiInfo;

typedef struct {
    int device;                   /* CUDA device ordinal (default 0) */
    int graph_iterations;         /* CFR iterations per captured CUDA graph (default 10) */
    float target_exploitability;  /* stop at this exploitability, % of pot; <= 0: run all iterations */
    int check_every;              /* iterations between exploitability checks (default 50) */
    int compute_exploitability;   /* 1: report the final exploitability in SSSolveStats */
} SSSolveOptions;

typedef struct {
    int iterations_run;
    double exploitability_pct;    /* NashConv / num_players / starting_pot * 100, FP64; -1 if not computed */
    double nashconv;              /* sum over players of best-response gain per unit of deal mass */
    double solve_ms;              /* device time of the CFR iterations */
    double node_hand_updates;     /* num_nodes x sum of hand counts x iterations */
    double queue_ms;              /* served form: submission until the request joined the running batch
                                     (admission and session build included); 0 for the other forms */
} SSSolveStats;

/* Served form: continuous batching of solve requests on one GPU. */
typedef struct {
    int device;                   /* CUDA device ordinal */
    double memory_budget_gb;      /* admit requests while their estimated device footprint fits */
    int block_iterations;         /* iterations between exploitability checks (default 25) */
    float target_exploitability;  /* retire a request at this exploitability, % of pot (default 0.5) */
    int max_iterations;           /* ... or after this many iterations (default 1000) */
    int graph_iterations;         /* iterations per captured CUDA graph (default 25) */
} SSServerOptions;
typedef struct SSServer SSServer;

/* A resident subgame: plan, device state and captured CUDA graphs stay on the
 * GPU between calls, so iterations can be added, the state reset or the
 * outputs read without re-uploading anything. */
typedef struct SSSession SSSession;

/* Per-kernel-class device time of one iteration (ss_session_profile). */
#define SS_PROFILE_CLASSES 8
typedef struct {
    int num_classes;
    char name[SS_PROFILE_CLASSES][16];
    int launches[SS_PROFILE_CLASSES];
    double ms[SS_PROFILE_CLASSES];       /* summed device time of the class in the iteration */
    double bytes[SS_PROFILE_CLASSES];    /* bytes the class must move in the iteration (minimum) */
    double iteration_ms;                 /* device time of the whole iteration */
} SSKernelProfile;

/* One launch of the profiled iteration (ss_session_profile_launches), in
 * launch order: its class (index into SSKernelProfile.name), the work items
 * it covers (decision nodes of one level, or terminals), device time and the
 * bytes it must move. */
typedef struct {
    int cls;
    int items;
    double ms;
    double bytes;
} SSLaunchRecord;

/* ── Host API ────────────────────────────────────────────────────────── */

#ifdef __cplusplus
extern "C" {
#endif

/* Build the betting tree for one street.  Replaces street_solve.cuh:172-178
 * (definition street_solve.cu:1192-1296): same node numbering, children
 * order, leaf numbering, BFS order and per-type index lists, with the
 * reference raise cap SS_MAX_RAISES.  Zeroes *tree_out first; the caller then
 * fills hands / weights / num_hands and, optionally, leaf_values and
 * frozen_action. */
int ss_build_tree(const int *board, int num_board,
                  int starting_pot, int effective_stack,
                  const float *bet_sizes, int num_bet_sizes,
                  int num_players, const int *acting_order,
                  int is_river, int use_cont_strats,
                  SSTreeData *tree_out);

/* Run max_iterations Linear-CFR iterations (every player traverses once per
 * iteration, in player order) on the GPU and fill *output.  Replaces
 * street_solve.cuh:186-190 (definition street_solve.cu:1298-1639).  Returns
 * SS_OK or a negative SS_ERR_* code; on failure *output is left zeroed and
 * nothing is leaked. */
int ss_solve_gpu(SSTreeData *tree_data, int max_iterations, SSOutput *output);

/* Free what ss_build_tree allocated (street_solve.cuh:192).  Unlike the
 * reference (street_solve.cu:1650) it does not free the caller-owned
 * leaf_values or frozen_action buffers. */
void ss_free_tree(SSTreeData *tree_data);

/* Free what ss_solve_gpu allocated (street_solve.cuh:193). */
void ss_free_output(SSOutput *output);

/* EXTENSION: layout of this build (which SS_MAX_HANDS the structs use). */
int ss_abi_info(SSAbiInfo *info);

/* EXTENSION: ss_build_tree with an explicit raise cap (the reference fixes it
 * at compile time, street_solve.cuh:42). */
int ss_build_tree_ex(const int *board, int num_board,
                     int starting_pot, int effective_stack,
                     const float *bet_sizes, int num_bet_sizes,
                     int num_players, const int *acting_order,
                     int is_river, int use_cont_strats, int max_raises,
                     SSTreeData *tree_out);

/* EXTENSION: default options. */
void ss_default_options(SSSolveOptions *opts);

/* EXTENSION: ss_solve_gpu with options (device, graph block, early stop at
 * an exploitability target) and statistics.  opts / stats may be NULL. */
int ss_solve_gpu_ex(SSTreeData *tree_data, int max_iterations,
                    const SSSolveOptions *opts, SSOutput *output, SSSolveStats *stats);

/* EXTENSION: FP64 exploitability of an average-strategy profile given in the
 * SSOutput layout ([num_decision_nodes][SS_MAX_ACTIONS][max_hands]) on the GPU.
 * br_value / cur_value (may be NULL) receive, per player, the best-response
 * and profile value summed over the player's hands weighted by range weight;
 * *deal_mass the valid-deal mass.  Returns SS_OK or SS_ERR_*. */
int ss_exploitability_gpu(const SSTreeData *tree_data, const float *avg_strategies,
                          double *exploitability_pct, double *nashconv,
                          double *br_value, double *cur_value, double *deal_mass);

/* EXTENSION: create a resident session for one subgame (copies everything it
 * needs; tree_data may be freed afterwards). */
int ss_session_create(const SSTreeData *tree_data, const SSSolveOptions *opts, SSSession **out);

/* EXTENSION: enqueue `iterations` more CFR iterations (asynchronous). */
int ss_session_run(SSSession *session, int iterations);

/* EXTENSION: wait for the session's queued work. */
int ss_session_synchronize(SSSession *session);

/* EXTENSION: back to iteration 0 (regrets, strategy sums and reach reset). */
int ss_session_reset(SSSession *session);

/* EXTENSION: iterations run since creation or the last reset. */
int ss_session_iterations(const SSSession *session);

/* EXTENSION: wait, then fill *output exactly as ss_solve_gpu would after the
 * same number of iterations (free it with ss_free_output). */
int ss_session_output(SSSession *session, SSOutput *output);

/* EXTENSION: run one more iteration as a graph with event nodes between the
 * kernel classes and report their device times and minimum bytes. */
int ss_session_profile(SSSession *session, SSKernelProfile *profile);

/* EXTENSION: the launches of the iteration the last ss_session_profile call
 * timed.  Writes at most max_records records and the launch count into
 * *num_records (either pointer may be NULL when max_records is 0). */
int ss_session_profile_launches(SSSession *session, SSLaunchRecord *records, int max_records, int *num_records);

/* EXTENSION: the CUDA stream (cudaStream_t) the session's kernels run on, so a
 * caller can order its own work or time the session with CUDA events. */
void *ss_session_stream(SSSession *session);

/* EXTENSION: FP64 exploitability of the session's current average strategy
 * (same outputs as ss_exploitability_gpu; any pointer may be NULL). */
int ss_session_exploitability(SSSession *session, double *exploitability_pct, double *nashconv,
                              double *br_value, double *cur_value, double *deal_mass);

/* EXTENSION (GPU form of the reference's between-street range update,
 * python/hud_solver.py:345-362 with python/range_narrowing.py:83-130):
 * narrow a range of num_hands entries (hand_cards [num_hands][2], weights
 * [num_hands], host arrays, weights updated in place) by the session's
 * current average strategy of `player` at decision node `node` (-1: the
 * player's first decision node, as get_avg_strategy reads it), for the action
 * label carried by the node's actions in action_mask (bit a = action a; the
 * last of them with a frequency above 0.001 counts, as in the reference's
 * label dictionary).  P(action | combo) is that frequency (0 at or below
 * 0.001); a combo the session's range does not hold (or an entry with
 * c0 > c1) gets 1 / max(number of distinct P values, 2); w' = w * P, raised
 * to 0.005 where w > 0, then divided by the largest w'.  FP64 throughout, bit
 * for bit the reference's Python.  *applied = 1 when some P is positive, else
 * 0 and the weights are left unchanged (the reference then falls back to
 * other sources).  The strategy sums are read where the solve left them;
 * nothing but the range crosses to the host. */
int ss_session_narrow(SSSession *session, int player, int node, unsigned int action_mask, int num_hands,
                      const int *hand_cards, double *weights, int *applied);

/* EXTENSION: release the session. */
void ss_session_destroy(SSSession *session);

/* EXTENSION: 7-card strengths of n hands (cards7 [n][7], cards 0..51) with
 * the device ranker, in the reference encoding (src/hand_eval.h:26-35). */
int ss_rank7_batch(const int *cards7, int n, unsigned int *strength_out);

/* EXTENSION: rank every 7-card set on the device; *checksum = sum over sets of
 * mix64(52-bit card mask) * strength (mod 2^64), category_counts[0..9] = sets
 * per category (may be NULL).  mix64 is the splitmix64 finaliser. */
int ss_rank7_checksum(unsigned long long *checksum, unsigned long long *category_counts);

/* EXTENSION (no counterpart in the reference): ss_solve_gpu for callers that
 * cannot allocate GPU memory at solve time -- e.g. a process whose device
 * memory belongs to another allocator, or a serving path with a
 * no-allocation policy.  It calls no CUDA allocation routine: all device
 * state lives in a 64 MiB static device array that every GPU loading this
 * library reserves until exit, and kernels run on the legacy default stream
 * without graphs or events.  The caller provides the output arrays in
 * *output: root_strategy (root actions x hands of the root player), root_ev
 * (num_players x max_hands), avg_strategies (num_decision_nodes x 8 x
 * max_hands) and avg_strategy_node_ids (num_decision_nodes); they are filled
 * like ss_solve_gpu's, and ss_free_output must not be called on them.  A
 * subgame whose state exceeds the array fails with SS_ERR_NOMEM and the size
 * it needs.  The first call on a device resolves the array's device address
 * (cudaGetSymbolAddress) and should come before any stream capture; the
 * address is kept for the life of the process, so a caller that destroys the
 * device's primary context (cudaDeviceReset) must not call this entry point
 * on that device afterwards.  All calls
 * share the array and it keeps the previous call's data (each call rewrites
 * what it reads); calls that overlap on the same GPU race. */
int ss_solve_gpu_noalloc(SSTreeData *tree_data, int max_iterations, SSOutput *output);

/* EXTENSION (batched form): solve n subgames of any size, street and player
 * count together -- each kernel launch covers one tree level of every
 * subgame.  With opts->target_exploitability > 0 each subgame is checked every
 * opts->check_every iterations and leaves the batch once its FP64
 * exploitability is at or below the target (or at max_iterations); otherwise
 * every subgame runs max_iterations.  outputs[i] / stats[i] (stats may be
 * NULL) are filled as by ss_solve_gpu_ex; free each output with
 * ss_free_output.  Per subgame, the arithmetic is the same as a solve alone. */
int ss_batch_solve(SSTreeData *const *trees, int n, int max_iterations, const SSSolveOptions *opts,
                   SSOutput *outputs, SSSolveStats *stats);

/* EXTENSION (served form): default server options. */
void ss_server_default_options(SSServerOptions *opts);

/* EXTENSION: start a server (a worker thread driving one batch on the device). */
int ss_server_create(const SSServerOptions *opts, SSServer **out);

/* EXTENSION: queue a solve request; the tree, ranges, leaf values and frozen
 * actions are copied, so the caller may free them on return. */
int ss_server_submit(SSServer *server, const SSTreeData *tree_data, long long *request_id);

/* EXTENSION: 0 = done (fills *output, free it with ss_free_output; *stats and
 * *latency_ms from submission to retirement, all optional), 1 = still queued
 * or running, < 0 = failed (the request is dropped). */
int ss_server_poll(SSServer *server, long long request_id, SSOutput *output, SSSolveStats *stats,
                   double *latency_ms);

/* EXTENSION: where a request stands without taking its result: *state 0 =
 * queued (not yet in the batch), 1 = in the batch, 2 = done (fetch it with
 * ss_server_poll / ss_server_wait); *iterations_run = CFR iterations it has
 * run so far (any pointer may be NULL).  Returns SS_OK, or SS_ERR_INVALID
 * for an unknown id, or the request's failure code. */
int ss_server_progress(SSServer *server, long long request_id, int *state, int *iterations_run);

/* EXTENSION: like ss_server_poll but blocks until the request is done. */
int ss_server_wait(SSServer *server, long long request_id, SSOutput *output, SSSolveStats *stats,
                   double *latency_ms);

/* EXTENSION: stop the worker and release the server (unfetched results too). */
void ss_server_destroy(SSServer *server);

/* ── Continuation values of a depth-limited subgame on the GPU ───────────
 *
 * Replaces the reference's Python producers compute_turn_leaf_values
 * (python/leaf_values.py:694-816) and compute_flop_leaf_equity
 * (python/leaf_values.py:408-571), which hud_solver.py calls before
 * ss_solve_gpu to fill SSTreeData.leaf_values.  Same result, bit for bit:
 * per runout, each hand's share of the opponent hand tuples it beats (ties
 * split 1/k), over tuples with no shared card, enumerated when there are at
 * most SS_LEAF_TUPLE_LIMIT of them and otherwise SS_LEAF_TUPLE_LIMIT drawn
 * with Python's random.Random(42) (python/leaf_values.py:573-691); averaged
 * over the runouts in the order given; then the first-order bias adjustment
 * at each leaf's pot for every one of the 4^N continuation profiles
 * (python/leaf_values.py:91-121), in FP64, stored as FP32. */

#define SS_LEAF_TUPLE_LIMIT 2000   /* python/leaf_values.py:615 */

typedef struct {
    int num_players;          /* 2 .. SS_MAX_PLAYERS */
    int max_hands;            /* row length of the output; >= every num_hands[p], <= 1326 */
    const int *num_hands;     /* [num_players] range sizes */
    const int *hand_cards;    /* [num_players][max_hands][2] cards 0..51 (rank * 4 + suit) */
    const int *board;         /* num_board cards: 3 (flop subgame) or 4 (turn subgame) */
    int num_board;
    const int *runout_cards;  /* [num_runouts][5 - num_board] cards completing the board, in averaging order */
    int num_runouts;
    const int *leaf_idx;      /* [num_leaves] LeafInfo.leaf_idx (index before the continuation expansion), >= 0 */
    const double *leaf_pot;   /* [num_leaves] LeafInfo.pot */
    int num_leaves;
} SSLeafValueInput;

/* EXTENSION (GPU form of python/leaf_values.py:694-816 and :408-571):
 * leaf_values [num_leaves * 4^num_players][num_players][max_hands] FP32,
 * laid out as the reference returns it and as SSTreeData.leaf_values reads
 * it; row leaf_idx * 4^N + profile of every leaf descriptor is written (a
 * later descriptor with the same leaf_idx wins, as in the reference loop),
 * every other entry is 0.  Returns SS_OK or a negative SS_ERR_* code. */
int ss_leaf_values_gpu(const SSLeafValueInput *input, float *leaf_values);

/* EXTENSION (host only, no GPU): the reference's opponent-tuple rule
 * (python/leaf_values.py:615-629) for opponents whose live-hand lists hold
 * list_sizes[0..num_opponents-1] hands: every tuple in itertools.product
 * order when their product is at most SS_LEAF_TUPLE_LIMIT, otherwise
 * SS_LEAF_TUPLE_LIMIT tuples drawn by random.Random(42).choice per opponent.
 * Writes positions into the lists, tuples[t * num_opponents + k], for at most
 * max_tuples tuples; returns the tuple count or a negative SS_ERR_* code. */
int ss_leaf_opponent_tuples(int num_opponents, const int *list_sizes, int *tuples, int max_tuples);

/* EXTENSION: message for the last failure on the calling thread ("" if none). */
const char *ss_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* B200_STREET_SOLVE_H */
