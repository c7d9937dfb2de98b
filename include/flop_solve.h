/*
 * flop_solve.h -- C ABI of the B200 multi-street (flop through river)
 * two-player Linear-CFR solver.
 *
 * Drop-in for the reference interface src/cuda/flop_solve.cuh: the structs
 * FSNode / FSTreeData / FSOutput keep the reference field order, types and
 * sizes byte for byte (flop_solve.cuh:45-114), and the entry points keep the
 * reference names, argument meaning and "0 on success" convention
 * (flop_solve.cuh:128-178), so the reference's ctypes callers
 * (bench/test_gpu_full_flop.py, bench/bench_gpu_flop.py,
 * precompute/run_all.py) bind this library unchanged.  Both builds of the
 * street solver library (libstreet_solve.so, libstreet_solve_wide.so) export
 * these entry points; the layout does not depend on SS_MAX_HANDS.
 */
#ifndef B200_FLOP_SOLVE_H
#define B200_FLOP_SOLVE_H

/* ── Limits (flop_solve.cuh:31-36) ───────────────────────────────────── */

#define FS_MAX_HANDS      200
#define FS_MAX_ACTIONS    6
#define FS_MAX_TREE_NODES 100000   /* informational, as in the reference (never enforced there) */
#define FS_MAX_BOARD      5

/* Node types (flop_solve.cuh:38-42) */
#define FS_NODE_DECISION  0
#define FS_NODE_FOLD      1
#define FS_NODE_SHOWDOWN  2
#define FS_NODE_CHANCE    3   /* deals the next board card: one child per card */

/* ── Flat tree node (flop_solve.cuh:45-56), 13 x int32 = 52 bytes ────── */

typedef struct {
    int type;            /* FS_NODE_* */
    int player;          /* acting player at decisions; winner at folds; -1 otherwise */
    int num_children;    /* decisions: actions; chance nodes: cards dealt */
    int first_child;     /* index into FSTreeData.children */
    int pot;             /* chips */
    int bets[2];         /* each player's bet this street */
    int board_cards[5];  /* the board at this node */
    int num_board;
} FSNode;

/* ── Solver input (flop_solve.cuh:60-83) ─────────────────────────────── */

typedef struct {
    FSNode *nodes;
    int *children;
    int num_nodes;
    int num_children_total;

    int hands[2][FS_MAX_HANDS][2];
    float weights[2][FS_MAX_HANDS];
    int num_hands[2];

    int *level_order;
    int *node_depth;
    int max_depth;

    int *decision_node_indices;
    int num_decision_nodes;

    int *showdown_node_indices;
    int num_showdown_nodes;
} FSTreeData;

/* ── Solver output (flop_solve.cuh:87-114) ───────────────────────────── */

typedef struct {
    float *root_strategy;       /* [root_num_actions][num_hands[root_player]], last iterate */
    int root_num_actions;
    int root_player;
    float *root_ev;             /* left NULL, as the reference leaves it */
    /* fs_solve_gpu_extract_all only: */
    float *all_avg_strategies;  /* [num_nodes][FS_MAX_ACTIONS][max_hands], decision nodes normalised */
    float *all_cfv;             /* [num_nodes][max_hands]: the last traverser's values at every node */
    int max_hands;
    int *turn_root_indices;     /* first decision node under each flop-end chance node */
    int *turn_root_cards;       /* the turn card dealt there */
    int num_turn_roots;
} FSOutput;

#ifdef __cplusplus
extern "C" {
#endif

/* Build the flop-through-river tree (flop_solve.cuh:128-135; definition
 * flop_solve.cu:894-972): the flop street with the given bet sizes, then the
 * turn and the river under every flop- and turn-ending chance node with a
 * single 0.75-pot bet size, one raise per street; same node numbering,
 * children order, BFS order and index lists as the reference.  Zeroes
 * *tree_out first; the caller then fills hands, weights and num_hands. */
int fs_build_tree(const int *flop_board, int starting_pot, int effective_stack,
                  const float *bet_sizes, int num_bet_sizes, FSTreeData *tree_out);

/* Run max_iterations Linear-CFR iterations (both players traverse, in
 * order) on the GPU and fill output->root_strategy / root_num_actions /
 * root_player (flop_solve.cuh:145-149; definition flop_solve.cu:974-1270).
 * Returns 0, or a negative SS_ERR_* code of street_solve.h with a message
 * from ss_last_error(); on failure *output is left zeroed. */
int fs_solve_gpu(FSTreeData *tree_data, int max_iterations, FSOutput *output);

/* fs_solve_gpu plus the normalised average strategy and the values of every
 * node, and the turn roots (flop_solve.cuh:168-176; definition
 * flop_solve.cu:1282-1572).  The reference re-runs the iterations for the
 * extraction; here the one solve's state is read out. */
int fs_solve_gpu_extract_all(FSTreeData *tree_data, int max_iterations, FSOutput *output);

/* Free what fs_build_tree allocated (flop_solve.cuh:152). */
void fs_free_tree(FSTreeData *tree_data);

/* Free what fs_solve_gpu / fs_solve_gpu_extract_all allocated (flop_solve.cuh:157). */
void fs_free_output(FSOutput *output);

#ifdef __cplusplus
}
#endif

#endif /* B200_FLOP_SOLVE_H */
