/*
 * ss_oracle.h -- CPU oracle for the single-street N-player Linear-CFR solver.
 *
 * TEST INFRASTRUCTURE ONLY: a plain-C restatement of the reference path
 * src/cuda/street_solve.cu (tree builder, hand strengths, level-batched CFR
 * kernels, output extraction), used by tests/, the smoke check and the CPU
 * baseline of bench.py as the checker.  It is never linked into, loaded by or
 * called from the product library.
 */
#ifndef SS_ORACLE_H
#define SS_ORACLE_H

#include <stdint.h>

#define ORC_MAX_PLAYERS 6
#define ORC_MAX_ACTIONS 8
#define ORC_NODE_DECISION 0
#define ORC_NODE_FOLD 1
#define ORC_NODE_SHOWDOWN 2
#define ORC_NODE_LEAF 4

/* Same 26-int field set and order as the reference SSNode
 * (src/cuda/street_solve.cuh:52-65), so node arrays compare byte for byte. */
typedef struct {
    int type;
    int player;
    int num_children;
    int first_child;
    int pot;
    int bets[ORC_MAX_PLAYERS];
    int board_cards[5];
    int num_board;
    int leaf_idx;
    int fold_player;
    int num_players;
    int active_players[ORC_MAX_PLAYERS];
} OrcNode;

typedef struct {
    OrcNode *nodes;
    int *children;
    int num_nodes;
    int num_children_total;
    int num_leaves;
    int num_players;
    int is_river;
    int starting_pot;
    int effective_stack;
    int board[5];
    int num_board;
    int *level_order; /* BFS order from node 0 */
    int *node_depth;
    int max_depth;
} OrcTree;

#ifdef __cplusplus
extern "C" {
#endif

int orc_build_tree(const int *board, int num_board, int starting_pot, int effective_stack,
                   const float *bet_sizes, int num_bet_sizes, int num_players,
                   const int *acting_order, int is_river, int use_cont_strats,
                   int max_raises, OrcTree *out);
void orc_free_tree(OrcTree *t);

uint32_t orc_eval7_cards(const int *cards7);
uint64_t orc_eval7_checksum(uint64_t *category_counts10);
void orc_eval7_many(const int *cards7, long n, uint32_t *out);

/* Solve with the reference semantics.  hands: [np][max_h][2], weights:
 * [np][max_h], num_hands: [np]; max_h = max(num_hands).  leaf_values:
 * [num_leaves][np][max_h] or NULL; frozen: [num_nodes] or NULL.
 * Outputs (any may be NULL): root_strategy [na_root][nh_root], root_ev [max_h],
 * avg_strategies [num_dec][8][max_h] with node ids [num_dec] (decision nodes
 * in index order), regrets / strategy_sum [num_nodes][8][max_h].  The f32
 * variant repeats the reference float arithmetic in the reference order; the
 * f64 variant performs the same steps in double precision. */
int orc_solve_f32(const OrcTree *t, const int *hands, const float *weights,
                  const int *num_hands, const float *leaf_values, const int *frozen,
                  int iterations, float *root_strategy, float *root_ev,
                  float *avg_strategies, int *avg_node_ids, float *regrets_out,
                  float *strategy_sum_out);
int orc_solve_f64(const OrcTree *t, const int *hands, const float *weights,
                  const int *num_hands, const float *leaf_values, const int *frozen,
                  int iterations, double *root_strategy, double *root_ev,
                  double *avg_strategies, int *avg_node_ids, double *regrets_out,
                  double *strategy_sum_out);

/* orc_solve_f64 with folds and leaves of one or two counted opponents
 * evaluated by the card-removal closed form (inclusion-exclusion over shared
 * cards, exact tuple counts for the reference's exact zeros) instead of the
 * odometer: the same sums in FP64, O(H * 52) per terminal and traverser hand
 * instead of O(H^2), so the full-size 3-player turn (1128 hands) is checkable.
 * Every other terminal is evaluated as in orc_solve_f64. */
int orc_solve_f64_closed(const OrcTree *t, const int *hands, const float *weights,
                         const int *num_hands, const float *leaf_values, const int *frozen,
                         int iterations, double *root_strategy, double *root_ev,
                         double *avg_strategies, int *avg_node_ids, double *regrets_out,
                         double *strategy_sum_out);

/* FP64 best-response exploitability of the average strategy profile given as
 * avg_strategies [num_dec][8][max_h] (decision nodes in index order).
 * Writes per-player best-response and profile values (sum over own hands of
 * weight x counterfactual value at the root) into br_value[np] / cur_value[np]
 * and the valid-deal mass into *deal_mass.  Returns NashConv / deal_mass.  */
double orc_exploitability(const OrcTree *t, const int *hands, const float *weights,
                          const int *num_hands, const float *leaf_values,
                          const int *frozen, const float *avg_strategies,
                          double *br_value, double *cur_value, double *deal_mass);

/* Counterfactual values of one traverser under a fixed profile (FP64):
 * cfv_root [max_h].  mode 0 = follow the profile at the traverser's nodes,
 * mode 1 = best response.  Exposed for the best-response parity tests. */
int orc_profile_cfv(const OrcTree *t, const int *hands, const float *weights,
                    const int *num_hands, const float *leaf_values, const int *frozen,
                    const float *avg_strategies, int traverser, int mode,
                    double *cfv_root);

#ifdef __cplusplus
}
#endif
#endif
