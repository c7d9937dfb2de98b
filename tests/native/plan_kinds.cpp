// Prints, as JSON, the terminal nodes of a tree and the planner's work-list
// sizes per traverser and terminal kind, for tests/test_plan_runs.py.
//   plan_kinds <players> <board cards (4 or 5)> <hands> <dup player or -1> <leaf values 0/1> <raises> [<bet sizes>]
// (bet sizes: 1 -> {1.0} (default), 2 -> {0.5, 1.0}, 3 -> {0.33, 0.75, 1.5})
// Turn trees get continuation leaves; each range is the first <hands>
// non-board combos in card order, with the first combo repeated for the
// dup player.
#include "ss_engine.h"
#include "street_solve.h"

#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

namespace ssb {
static std::string g_err;
void set_error(const std::string &s) { g_err = s; }
const char *last_error() { return g_err.c_str(); }
}  // namespace ssb

int main(int argc, char **argv) {
    if (argc != 7 && argc != 8) return 2;
    const int np = std::atoi(argv[1]), nb = std::atoi(argv[2]), nh = std::atoi(argv[3]);
    const int dup = std::atoi(argv[4]), with_leaves = std::atoi(argv[5]), raises = std::atoi(argv[6]);
    const int board[5] = {0, 13, 26, 40, 51};
    const int nbets = argc == 8 ? std::atoi(argv[7]) : 1;
    if (nbets < 1 || nbets > 3) return 2;
    const float bet_sets[3][3] = {{1.0f}, {0.5f, 1.0f}, {0.33f, 0.75f, 1.5f}};
    const float *bets = bet_sets[nbets - 1];
    int order[SS_MAX_PLAYERS];
    for (int p = 0; p < np; ++p) order[p] = p;
    const bool river = nb == 5;
    ssb::BuiltTree bt;
    if (ssb::build_street_tree(board, nb, 100, 400, bets, nbets, np, order, river ? 1 : 0, river ? 0 : 1, raises, &bt) !=
        SS_OK)
        return 3;
    std::vector<int> base;
    for (int a = 0; a < 52 && static_cast<int>(base.size()) < 2 * nh; ++a)
        for (int b = a + 1; b < 52 && static_cast<int>(base.size()) < 2 * nh; ++b) {
            bool on = false;
            for (int i = 0; i < nb; ++i) on = on || board[i] == a || board[i] == b;
            if (!on) {
                base.push_back(a);
                base.push_back(b);
            }
        }
    std::vector<int> hands[SS_MAX_PLAYERS];
    std::vector<float> w[SS_MAX_PLAYERS];
    for (int p = 0; p < np; ++p) {
        hands[p] = base;
        if (p == dup) {
            hands[p][2] = hands[p][0];
            hands[p][3] = hands[p][1];
        }
        w[p].assign(hands[p].size() / 2, 0.5f);
    }
    const int mh = nh;
    std::vector<float> lv(static_cast<size_t>(bt.num_leaves) * np * mh, 0.25f);
    ssb::Problem pb{};
    pb.nodes = bt.nodes.data();
    pb.children = bt.children.data();
    pb.num_nodes = static_cast<int>(bt.nodes.size());
    pb.num_children_total = static_cast<int>(bt.children.size());
    pb.num_players = np;
    for (int p = 0; p < np; ++p) {
        pb.hands[p] = hands[p].data();
        pb.weights[p] = w[p].data();
        pb.num_hands[p] = static_cast<int>(w[p].size());
    }
    for (int i = 0; i < nb; ++i) pb.board[i] = board[i];
    pb.num_board = nb;
    pb.is_river = river ? 1 : 0;
    pb.starting_pot = 100;
    if (with_leaves && bt.num_leaves > 0) {
        pb.leaf_values = lv.data();
        pb.num_leaves = bt.num_leaves;
    }
    ssb::Plan P;
    const int rc = ssb::build_plan(pb, &P);
    std::printf("{\"rc\": %d, \"dup\": [", rc);
    for (int p = 0; p < np; ++p) std::printf("%s%d", p ? ", " : "", rc == SS_OK ? P.dup[p] : -1);
    std::printf("], \"hands\": [");
    for (int p = 0; p < np; ++p) std::printf("%s%d", p ? ", " : "", rc == SS_OK ? P.H[p] : -1);
    std::printf("], \"terminals\": [");
    bool first = true;
    for (size_t x = 0; x < bt.nodes.size(); ++x) {
        const SSNode &n = bt.nodes[x];
        if (n.type == SS_NODE_DECISION) continue;
        std::printf("%s[%d, %d, [", first ? "" : ", ", n.type, n.leaf_idx);
        for (int p = 0; p < np; ++p) std::printf("%s%d", p ? ", " : "", n.active_players[p]);
        std::printf("]]");
        first = false;
    }
    std::printf("], \"kinds\": [");
    for (int t = 0; t < np; ++t) {
        std::printf("%s[", t ? ", " : "");
        for (int k = 0; k < ssb::TK_COUNT; ++k)
            std::printf("%s%zu", k ? ", " : "", rc == SS_OK ? P.term[t][k].size() : static_cast<size_t>(0));
        std::printf("]");
    }
    // closed-form groups: per traverser and kind (CR1, CR2, CR3), every item
    // as [gextra, follow, rows 0..2, players 0..2]
    std::printf("], \"groups\": [");
    for (int t = 0; t < np; ++t) {
        std::printf("%s[", t ? ", " : "");
        int kk = 0;
        for (int kind : {ssb::TK_CR1, ssb::TK_CR2, ssb::TK_CR3}) {
            std::printf("%s[", kk++ ? ", " : "");
            if (rc == SS_OK)
                for (size_t i = 0; i < P.term[t][kind].size(); ++i) {
                    const ssb::TermItem &it = P.term[t][kind][i];
                    std::printf("%s[%d, %d, %d, %d, %d, %d, %d, %d]", i ? ", " : "", it.gextra, it.follow,
                                it.opp_row[0], it.opp_row[1], it.opp_row[2], it.opp_player[0], it.opp_player[1],
                                it.opp_player[2]);
                }
            std::printf("]");
        }
        std::printf("]");
    }
    // value/regret items with an inline frontier: rows and per-edge ends
    // decode to the frontier tables (bad = mismatches), and every frontier
    // short enough is inline
    int inl = 0, bad = 0;
    if (rc == SS_OK)
        for (int t = 0; t < np; ++t)
            for (const auto &lv : P.cfv_levels[t])
                for (const ssb::CfvItem &it : lv) {
                    const int k0 = P.fr_off[it.first_edge], n = P.fr_off[it.first_edge + it.na] - k0;
                    if ((n <= ssb::kCfvInline) != (it.nfr == n)) ++bad;
                    if (it.nfr == 0) continue;
                    ++inl;
                    for (int i = 0; i < n; ++i) {
                        if (it.fr[i] != P.fr_items[k0 + i]) ++bad;
                        int e = 0;
                        for (int a = 0; a < SS_MAX_ACTIONS - 1; ++a)
                            e += i > static_cast<int>((static_cast<unsigned>(it.fr_bnd) >> (4 * a)) & 15u) ? 1 : 0;
                        if (!(P.fr_off[it.first_edge + e] <= k0 + i && k0 + i < P.fr_off[it.first_edge + e + 1])) ++bad;
                    }
                }
    std::printf("], \"cfv_inline\": [%d, %d", inl, bad);
    // launch heads: per traverser, [CR1 heads (none), CR2 heads]
    std::printf("], \"heads\": [");
    for (int t = 0; t < np; ++t) {
        std::printf("%s[", t ? ", " : "");
        int kk = 0;
        for (int kind : {ssb::TK_CR1, ssb::TK_CR2}) {
            std::printf("%s[", kk++ ? ", " : "");
            if (rc == SS_OK)
                for (size_t i = 0; i < P.term_heads[t][kind].size(); ++i)
                    std::printf("%s%d", i ? ", " : "", P.term_heads[t][kind][i]);
            std::printf("]");
        }
        std::printf("]");
    }
    // two-opponent chains: per traverser, every item's [chain, chained]
    std::printf("], \"chains\": [");
    for (int t = 0; t < np; ++t) {
        std::printf("%s[", t ? ", " : "");
        if (rc == SS_OK)
            for (size_t i = 0; i < P.term[t][ssb::TK_CR2].size(); ++i) {
                const ssb::TermItem &it = P.term[t][ssb::TK_CR2][i];
                std::printf("%s[%d, %d]", i ? ", " : "", it.chain, it.chained);
            }
        std::printf("]");
    }
    std::printf("]}\n");
    return 0;
}
