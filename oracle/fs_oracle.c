/*
 * fs_oracle.c -- CPU oracle for the multi-street (flop through river)
 * two-player Linear-CFR solver.
 *
 * TEST INFRASTRUCTURE ONLY: a plain-C restatement of the reference's
 * src/cuda/flop_solve.cu solve (:974-1270, extraction :1282-1572) on a tree
 * built by fs_build_tree (whose layout include/flop_solve.h fixes), used by
 * tests/ as the checker; the product library never loads it.  The CFR body
 * is compiled twice: in float, the reference's arithmetic in its order --
 * including the multiply-adds the GPU compiler fuses in the reference's
 * kernels, written here as fmaf -- and in double.  It is pinned to the
 * reference's own GPU build by fixtures (tests/golden/make_flop_golden.py).
 *
 *   per iteration t = 1..T, per traverser (0 then 1):
 *     regret matching at every decision node                 :652-684
 *     the opponent's reach from its weights, level by level  :686-729
 *     fold and showdown values                               :731-833
 *     values bottom-up by level: the traverser's nodes update regrets
 *     (r += v_a - v, r *= t / (t + 1)) and strategy sums (s += t sigma),
 *     chance nodes average their children                   :835-892
 *   outputs: the last regret-matched strategy at node 0; the normalised
 *   strategy sums and the last pass's values at every node.
 */
#include "oracle_eval.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define FSO_MAX_HANDS 200
#define FSO_MAX_ACTIONS 6

typedef struct {
    int type, player, num_children, first_child, pot;
    int bets[2];
    int board_cards[5];
    int num_board;
} FsoNode;

#define REAL float
#define FSUF(n) n##_f32
#define FLIT(x) x##f
#define FMA(a, b, c) fmaf((a), (b), (c))
#include "fs_oracle_impl.h"
#undef REAL
#undef FSUF
#undef FLIT
#undef FMA

#define REAL double
#define FSUF(n) n##_f64
#define FLIT(x) x
#define FMA(a, b, c) fma((a), (b), (c))
#include "fs_oracle_impl.h"
#undef REAL
#undef FSUF
#undef FLIT
#undef FMA
