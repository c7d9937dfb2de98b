// fs_engine.h -- internal interface of the multi-street (flop through river)
// two-player solver: tree builder (fs_tree.cpp), planner and GPU solve
// (fs_engine.cu).  The C ABI (fs_abi.cpp) is include/flop_solve.h.
#pragma once

#include "flop_solve.h"
#include "ss_engine.h"

#include <vector>

namespace ssb {
namespace fs {

int build_tree(const int *flop, int starting_pot, int effective_stack, const float *sizes, int num_sizes,
               FSTreeData *out);
void free_tree(FSTreeData *t);

// One terminal for one traverser.  Folds pay `payoff` times the opponent's
// reach over hands sharing no card with the traverser's hand or the node's
// board; showdowns pay +-half_pot per opponent hand by the 7-card strengths
// on board `sboard` (ties 0, a hand the board blocks 0).  The value row is
// stored times `scale`: the product of 1 / cards dealt over the chance nodes
// between the terminal and the traverser's edge whose frontier holds it.
struct alignas(16) FsTermItem {
    int node;
    int kind;          // 0 fold, 1 showdown
    int opp_row;       // the opponent's sequence (reach row) at the node
    int sboard;        // showdown: row of the strength table
    float payoff;      // fold
    float half_pot;    // showdown
    float scale;
    int nb;            // board cards at the node
    int board[5];
    int pad_[3];
};

struct FsPlan {
    int N = 0, E = 0, HS = 0, max_h = 0;
    int H[2] = {0, 0};
    int root_player = 0, root_na = 0;
    std::vector<int> first_edge, edge_node, dec_nodes;
    std::vector<std::vector<ReachItem>> reach_levels[2];
    std::vector<std::vector<CfvItem>> cfv_levels[2];
    std::vector<int> cfv_nlong[2];
    std::vector<int> fr_off, fr_items;
    std::vector<FsTermItem> term[2];   // per traverser: folds, then showdowns
    int nfold[2] = {0, 0};
    std::vector<int> sboards;          // [nsb][5] river boards of the showdowns
    std::vector<int> hand_cards;       // [2][HS]: c0 | c1 << 8, -1 padding
    std::vector<int> f_coff, f_clist;  // [2][53], [2][2 * HS]: each player's hands holding card c
    // showdown tables per river board b and player p, [nsb][2][...]:
    //   ord  [HS]   hand index at each position of ascending strength (board-
    //               blocked hands, strength 0, first), -1 past the range
    //   hpos [HS]   per hand (as traverser): int4 {lo | hi << 16, c1 | c2 << 8,
    //               l1lo | l1hi << 16, l2lo | l2hi << 16} -- the opponent's
    //               positions below its strength (lo) and up to it (hi), and the
    //               same counts within the opponent's list of each of its cards
    //   coff [53]   the opponent p's card lists: hands holding card c at
    //   clist[2*HS] clist[coff[c] .. coff[c+1]), by position
    std::vector<int> sd_ord, sd_hpos, sd_coff, sd_clist;
    std::vector<unsigned> sd_str;      // [nsb][2][HS] strengths (0: blocked / padding)
    std::vector<int> depth_nodes;      // read-out: nodes by BFS depth, deepest level first
    std::vector<int> depth_off;        // [levels + 1]
};

int build_plan(const FSTreeData &td, FsPlan *plan);

// extract: also fill all_avg_strategies, all_cfv and the turn roots
int solve(FSTreeData *td, int iterations, FSOutput *out, bool extract);
void free_output(FSOutput *out);

}  // namespace fs
}  // namespace ssb
