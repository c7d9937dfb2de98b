// ss_plan.cpp -- host planner: validates one subgame and flattens it into the
// work lists the kernels consume.
//
// Layout decisions (all rows are HS floats, HS = max hands rounded up to 32):
//   * every decision-node edge e (= node, action) owns one row of regrets,
//     strategy sums and reach; the reach row of e holds the acting player's
//     reach after taking that action, so a player's reach at any node is the
//     row of the last edge that player took on the path from the root (or the
//     player's range weights, rows E .. E + np - 1, before it acted).  Reach
//     is therefore stored once per sequence, not once per node and player as
//     in the reference (street_solve.cu:1315-1337).
//   * values: one row per node; only terminals and the current traverser's
//     decision nodes are written.  The value of a traverser edge is the sum of
//     the rows of its frontier: the terminals and traverser nodes reached
//     through other players' decisions, which only sum their children
//     (street_solve.cu:1176-1184).
//   * reach is propagated top-down per player, level by level in that
//     player's own decision depth; values and regrets are updated bottom-up
//     per traverser, level by level in the traverser's own decision height.
#include "ss_engine.h"
#include "ss_rank.cuh"

#include <algorithm>
#include <cstring>
#include <string>

namespace ssb {

uint32_t rank7_host(const int *board5, int c0, int c1) {
    int c[7] = {board5[0], board5[1], board5[2], board5[3], board5[4], c0, c1};
    for (int i = 0; i < 7; ++i)
        for (int j = i + 1; j < 7; ++j)
            if (c[i] == c[j]) return 0;
    return rank7(c);
}

namespace {

bool fail(const std::string &m) {
    set_error(m);
    return false;
}

bool validate(const Problem &pb, Plan &P) {
    if (!pb.nodes || !pb.children || pb.num_nodes < 1)
        return fail("tree has no nodes");
    if (pb.num_players < 1 || pb.num_players > SS_MAX_PLAYERS)
        return fail("num_players must be 1..6");
    P.np = pb.num_players;
    P.N = pb.num_nodes;
    P.max_h = 0;
    for (int p = 0; p < P.np; ++p) {
        if (pb.num_hands[p] < 0) return fail("negative hand count");
        if (pb.num_hands[p] > 0 && (!pb.hands[p] || !pb.weights[p])) return fail("missing range");
        P.H[p] = pb.num_hands[p];
        P.max_h = std::max(P.max_h, P.H[p]);
        for (int h = 0; h < P.H[p]; ++h) {
            int a = pb.hands[p][2 * h], b = pb.hands[p][2 * h + 1];
            if (a < 0 || a > 51 || b < 0 || b > 51 || a == b)
                return fail("hand " + std::to_string(h) + " of player " + std::to_string(p) +
                            " is not two distinct cards 0..51");
        }
    }
    if (P.max_h == 0) return fail("every range is empty");
    for (int i = 0; i < P.N; ++i) {
        const SSNode &n = pb.nodes[i];
        if (n.type == SS_NODE_DECISION) {
            if (n.num_children < 1 || n.num_children > SS_MAX_ACTIONS)
                return fail("decision node " + std::to_string(i) + " has " +
                            std::to_string(n.num_children) + " actions (1..8 supported)");
            if (n.player < 0 || n.player >= P.np)
                return fail("decision node " + std::to_string(i) + " has no valid player");
            if (n.first_child < 0 || n.first_child + n.num_children > pb.num_children_total)
                return fail("decision node " + std::to_string(i) + " children out of range");
            for (int a = 0; a < n.num_children; ++a) {
                int c = pb.children[n.first_child + a];
                if (c <= 0 || c >= P.N) return fail("child id out of range");
            }
        } else if (n.type == SS_NODE_FOLD || n.type == SS_NODE_SHOWDOWN || n.type == SS_NODE_LEAF) {
            if (n.num_children != 0) return fail("terminal node with children");
            if (n.type == SS_NODE_FOLD && (n.player < 0 || n.player >= P.np))
                return fail("fold node without a winner");
            if (n.type == SS_NODE_LEAF && pb.leaf_values &&
                (n.leaf_idx >= pb.num_leaves))
                return fail("leaf_idx beyond num_leaves");
        } else {
            return fail("unknown node type");
        }
        for (int p = 0; p < P.np; ++p)
            if (n.bets[p] < 0) return fail("negative bet");
        if (n.num_board != pb.nodes[0].num_board) return fail("nodes disagree on the board");
        for (int b = 0; b < n.num_board && b < 5; ++b)
            if (n.board_cards[b] != pb.nodes[0].board_cards[b]) return fail("nodes disagree on the board");
    }
    if (pb.frozen)
        for (int i = 0; i < P.N; ++i)
            if (pb.frozen[i] >= SS_MAX_ACTIONS) return fail("frozen action index too large");
    return true;
}

}  // namespace

void inline_frontier(CfvItem &it, const std::vector<int> &fr_off, const std::vector<int> &fr_items) {
    const int k0 = fr_off[it.first_edge], n = fr_off[it.first_edge + it.na] - k0;
    it.nfr = 0;
    it.fr_bnd = 0;
    if (n <= 0 || n > kCfvInline || it.na > SS_MAX_ACTIONS) return;
    unsigned bnd = 0;
    for (int a = 0; a < SS_MAX_ACTIONS; ++a)
        bnd |= static_cast<unsigned>(a < it.na ? fr_off[it.first_edge + a + 1] - k0 - 1 : 15) << (4 * a);
    for (int i = 0; i < n; ++i) it.fr[i] = fr_items[k0 + i];
    it.nfr = n;
    it.fr_bnd = static_cast<int>(bnd);
}

int build_plan(const Problem &pb, Plan *out) {
    Plan &P = *out;
    if (!validate(pb, P)) return SS_ERR_INVALID;
    const int np = P.np, N = P.N;
    const SSNode *nd = pb.nodes;
    P.HS = (P.max_h + 31) / 32 * 32;

    // breadth-first order; the tree must be a rooted tree over all nodes
    std::vector<int> order;
    order.reserve(N);
    std::vector<int> parent(N, -2), parent_act(N, -1);
    order.push_back(0);
    parent[0] = -1;
    for (size_t q = 0; q < order.size(); ++q) {
        const int x = order[q];
        if (nd[x].type != SS_NODE_DECISION) continue;
        for (int a = 0; a < nd[x].num_children; ++a) {
            const int c = pb.children[nd[x].first_child + a];
            if (parent[c] != -2) {
                set_error("node " + std::to_string(c) + " is reached twice: not a tree");
                return SS_ERR_INVALID;
            }
            parent[c] = x;
            parent_act[c] = a;
            order.push_back(c);
        }
    }
    if (static_cast<int>(order.size()) != N) {
        set_error("some nodes are not reachable from node 0");
        return SS_ERR_INVALID;
    }
    if (nd[0].type != SS_NODE_DECISION) {
        set_error("node 0 must be a decision node");
        return SS_ERR_INVALID;
    }
    P.root_player = nd[0].player;
    P.root_na = nd[0].num_children;
    P.starting_pot = pb.starting_pot;

    // edges in BFS order
    P.first_edge.assign(N, -1);
    P.edge_node.clear();
    for (int x : order)
        if (nd[x].type == SS_NODE_DECISION) {
            P.first_edge[x] = static_cast<int>(P.edge_node.size());
            for (int a = 0; a < nd[x].num_children; ++a) P.edge_node.push_back(x);
        }
    P.E = static_cast<int>(P.edge_node.size());
    const int E = P.E;
    P.dec_nodes.clear();
    for (int i = 0; i < N; ++i)
        if (nd[i].type == SS_NODE_DECISION) P.dec_nodes.push_back(i);
    P.num_dec = static_cast<int>(P.dec_nodes.size());

    // last edge of each player on the path to each node, and own-decision depth
    std::vector<int> last(static_cast<size_t>(N) * np), pdepth(static_cast<size_t>(N) * np, 0);
    for (int x : order) {
        for (int p = 0; p < np; ++p) {
            int v, d;
            if (x == 0) {
                v = E + p;
                d = 0;
            } else {
                const int par = parent[x];
                const bool acted = nd[par].player == p;
                v = acted ? P.first_edge[par] + parent_act[x] : last[static_cast<size_t>(par) * np + p];
                d = pdepth[static_cast<size_t>(par) * np + p] + (acted ? 1 : 0);
            }
            last[static_cast<size_t>(x) * np + p] = v;
            pdepth[static_cast<size_t>(x) * np + p] = d;
        }
    }
    auto frozen_of = [&](int x) { return pb.frozen ? pb.frozen[x] : -1; };

    // reach levels per player (own-decision depth, top-down)
    for (int p = 0; p < np; ++p) {
        P.reach_levels[p].clear();
        for (int x : order) {
            if (nd[x].type != SS_NODE_DECISION || nd[x].player != p) continue;
            const int lev = pdepth[static_cast<size_t>(x) * np + p];
            if (static_cast<int>(P.reach_levels[p].size()) <= lev) P.reach_levels[p].resize(lev + 1);
            ReachItem it;
            it.first_edge = P.first_edge[x];
            it.na = nd[x].num_children;
            it.parent_row = last[static_cast<size_t>(x) * np + p];
            it.frozen = frozen_of(x);
            P.reach_levels[p][lev].push_back(it);
        }
    }

    // frontiers: per edge, the terminals / same-player nodes reached through
    // other players' decisions, in depth-first child order
    P.fr_off.assign(E + 1, 0);
    P.fr_items.clear();
    std::vector<int> stack;
    auto collect = [&](int start, int p, std::vector<int> &dst) {
        stack.clear();
        stack.push_back(start);
        while (!stack.empty()) {
            const int x = stack.back();
            stack.pop_back();
            if (nd[x].type != SS_NODE_DECISION || nd[x].player == p) {
                dst.push_back(x);
                continue;
            }
            for (int a = nd[x].num_children - 1; a >= 0; --a)
                stack.push_back(pb.children[nd[x].first_child + a]);
        }
    };
    for (int e = 0; e < E; ++e) {
        const int x = P.edge_node[e];
        const int a = e - P.first_edge[x];
        collect(pb.children[nd[x].first_child + a], nd[x].player, P.fr_items);
        P.fr_off[e + 1] = static_cast<int>(P.fr_items.size());
    }
    for (int p = 0; p < np; ++p) {
        P.root_fr[p].clear();
        collect(0, p, P.root_fr[p]);
    }

    // cfv levels per traverser: height in own decisions (bottom-up)
    std::vector<int> height(N, 0);
    for (int t = 0; t < np; ++t) {
        P.cfv_levels[t].clear();
        for (int q = N - 1; q >= 0; --q) {
            const int x = order[q];
            if (nd[x].type != SS_NODE_DECISION || nd[x].player != t) continue;
            int h = 0;
            const int fe = P.first_edge[x];
            for (int k = P.fr_off[fe]; k < P.fr_off[fe + nd[x].num_children]; ++k) {
                const int y = P.fr_items[k];
                if (nd[y].type == SS_NODE_DECISION) h = std::max(h, height[y] + 1);
            }
            height[x] = h;
            if (static_cast<int>(P.cfv_levels[t].size()) <= h) P.cfv_levels[t].resize(h + 1);
            CfvItem it;
            it.first_edge = fe;
            it.na = nd[x].num_children;
            it.frozen = frozen_of(x);
            it.node = x;
            inline_frontier(it, P.fr_off, P.fr_items);
            P.cfv_levels[t][h].push_back(it);
        }
        P.cfv_nlong[t].assign(P.cfv_levels[t].size(), 0);
        for (size_t l = 0; l < P.cfv_levels[t].size(); ++l) {
            P.cfv_nlong[t][l] = order_cfv_level(P.cfv_levels[t][l], [&](const CfvItem &it) {
                return P.fr_off[it.first_edge + it.na] - P.fr_off[it.first_edge];
            });
        }
    }

    // board and hand tables
    const int nb = nd[0].num_board;
    const int *board = nd[0].board_cards;
    bool on_board[52] = {};
    for (int b = 0; b < nb && b < 5; ++b)
        if (board[b] >= 0 && board[b] < 52) on_board[board[b]] = true;
    const size_t HS = static_cast<size_t>(P.HS);
    int dense[52];
    P.deck = 0;
    for (int x = 0; x < 52; ++x) dense[x] = on_board[x] ? 63 : P.deck++;
    P.hand_code.assign(static_cast<size_t>(np) * HS, -1);
    for (int p = 0; p < np; ++p)
        for (int h = 0; h < P.H[p]; ++h) {
            const int a = pb.hands[p][2 * h], b = pb.hands[p][2 * h + 1];
            const int blocked = (on_board[a] || on_board[b]) ? 1 : 0;
            P.hand_code[p * HS + h] = a | (b << 8) | (blocked << 16) | (dense[a] << 20) | (dense[b] << 26);
        }

    // ranges holding the same combo twice need atomic accumulation in the
    // terminal kernels' combo tables
    for (int p = 0; p < np; ++p) {
        std::vector<char> seen(52 * 52, 0);
        P.dup[p] = 0;
        for (int h = 0; h < P.H[p]; ++h) {
            int a = pb.hands[p][2 * h], b = pb.hands[p][2 * h + 1];
            if (a > b) std::swap(a, b);
            if (seen[a * 52 + b]++) P.dup[p] = 1;
        }
    }

    // terminal work lists per traverser
    bool need_sd = false;
    P.enum_work = 0;
    for (int t = 0; t < np; ++t)
        for (int k = 0; k < TK_COUNT; ++k) P.term[t][k].clear();
    for (int x = 0; x < N; ++x) {
        const SSNode &n = nd[x];
        if (n.type == SS_NODE_DECISION) continue;
        for (int t = 0; t < np; ++t) {
            TermItem it;
            std::memset(&it, 0, sizeof(it));
            it.node = x;
            it.leaf_off = -1;
            int kind = TK_ZERO;
            int k = 0;
            auto add_opp = [&](int o) {
                it.opp_row[k] = last[static_cast<size_t>(x) * np + o];
                it.opp_player[k] = o;
                ++k;
            };
            // three counted opponents: closed form for large ranges without
            // repeated combos in the two that form its matrices
            auto multi = [&]() {
                if (k != 3 || P.dup[it.opp_player[0]] || P.dup[it.opp_player[1]]) return static_cast<int>(TK_ENUM);
                for (int i = 0; i < 3; ++i)
                    if (P.H[it.opp_player[i]] < kCr3MinHands) return static_cast<int>(TK_ENUM);
                return static_cast<int>(TK_CR3);
            };
            if (n.type == SS_NODE_FOLD) {
                for (int o = 0; o < np; ++o)
                    if (o != t) add_opp(o);
                it.payoff = (n.player == t) ? static_cast<float>(n.pot - n.bets[t])
                                            : -static_cast<float>(n.bets[t]);
                it.kind_detail = 0;
                kind = k == 0 ? TK_LEAF0 : k == 1 ? (P.dup[it.opp_player[0]] ? TK_CR1D : TK_CR1) : k == 2 ? TK_CR2 : multi();
            } else if (n.type == SS_NODE_LEAF) {
                if (pb.leaf_values && n.leaf_idx >= 0) {
                    for (int o = 0; o < np; ++o)
                        if (o != t && n.active_players[o]) add_opp(o);
                    it.leaf_off = (n.leaf_idx * np + t) * P.max_h;
                    it.kind_detail = 1;
                    kind = k == 0 ? TK_LEAF0 : k == 1 ? (P.dup[it.opp_player[0]] ? TK_CR1D : TK_CR1) : k == 2 ? TK_CR2 : multi();
                }
            } else {  // showdown
                if (pb.is_river && n.active_players[t]) {
                    for (int o = 0; o < np; ++o)
                        if (o != t && n.active_players[o]) add_opp(o);
                    it.pot = static_cast<float>(n.pot);
                    it.bet = static_cast<float>(n.bets[t]);
                    it.kind_detail = 2;
                    const bool nodup = !P.dup[t] && !P.dup[it.opp_player[0]] && !P.dup[it.opp_player[1]];
                    bool large = k == 3;
                    for (int i = 0; i < k && large; ++i) large = P.H[it.opp_player[i]] >= kCr3MinHands;
                    kind = k == 1 ? TK_SD1 : (k == 2 && nodup) ? TK_SD2 : (large && nodup) ? TK_SD3 : TK_ENUM;
                    need_sd = true;
                }
            }
            it.k = k;
            if (kind == TK_ENUM) {
                double w = P.H[t];
                for (int i = 0; i < k; ++i) w *= std::max(1, P.H[it.opp_player[i]]);
                P.enum_work += w;
            }
            P.term[t][kind].push_back(it);
        }
    }

    // one-, two- and three-opponent terminals sharing their opponents' reach
    // rows share their card-removal mass: order them by the rows and mark
    // groups (rows and players past the counted ones are 0)
    for (int t = 0; t < np; ++t)
        for (int kind : {TK_CR1, TK_CR2, TK_CR3}) {
            std::vector<TermItem> &v = P.term[t][kind];
            std::stable_sort(v.begin(), v.end(), [](const TermItem &u, const TermItem &w) {
                if (u.opp_row[0] != w.opp_row[0]) return u.opp_row[0] < w.opp_row[0];
                if (u.opp_row[1] != w.opp_row[1]) return u.opp_row[1] < w.opp_row[1];
                return u.opp_row[2] < w.opp_row[2];
            });
            auto same = [](const TermItem &u, const TermItem &w) {
                for (int i = 0; i < 3; ++i)
                    if (u.opp_row[i] != w.opp_row[i] || u.opp_player[i] != w.opp_player[i]) return false;
                return true;
            };
            for (size_t i = 0; i < v.size();) {
                size_t j = i + 1;
                while (j < v.size() && j - i < static_cast<size_t>(kTermGroupMax) && same(v[j], v[i]))
                    ++j;
                v[i].gextra = static_cast<int>(j - i - 1);
                for (size_t m = i + 1; m < j; ++m) v[m].follow = 1;
                i = j;
            }
        }

    // two-opponent chains: groups on the same first-opponent row, as many per
    // chain as keep the launch at kCr2ChainBlocks blocks or more
    for (int t = 0; t < np; ++t) {
        std::vector<TermItem> &v = P.term[t][TK_CR2];
        std::vector<size_t> leads;
        for (size_t i = 0; i < v.size(); i += static_cast<size_t>(v[i].gextra) + 1) leads.push_back(i);
        const int len = std::min(kCr2ChainMax, std::max(1, static_cast<int>(leads.size()) / kCr2ChainBlocks));
        if (len < 2) continue;
        for (size_t g = 0; g < leads.size();) {
            const TermItem &h = v[leads[g]];
            size_t e = g + 1;
            while (e < leads.size() && static_cast<int>(e - g) < len && v[leads[e]].opp_row[0] == h.opp_row[0] &&
                   v[leads[e]].opp_player[0] == h.opp_player[0] && v[leads[e]].opp_player[1] == h.opp_player[1])
                ++e;
            v[leads[g]].chain = static_cast<int>(e - g - 1);
            for (size_t m = g + 1; m < e; ++m) v[leads[m]].chained = 1;
            g = e;
        }
    }
    for (int t = 0; t < np; ++t)
        for (int k = 0; k < TK_COUNT; ++k) {
            P.term_heads[t][k].clear();
            if (k != TK_CR2) continue;
            const std::vector<TermItem> &v = P.term[t][k];
            for (size_t i = 0; i < v.size(); ++i)
                if (!v[i].follow && !v[i].chained) P.term_heads[t][k].push_back(static_cast<int>(i));
        }

    // showdown tables: every non-board combo ranked on the 5-card board
    P.ncomb = 0;
    P.sd_combo.clear();
    P.sd_card_list.assign(52 * 52, -1);
    P.sd_card_partner.assign(52 * 52, -1);
    P.sd_pos.assign(static_cast<size_t>(np) * HS, -1);
    P.pos_hand.clear();
    P.sd_seg.clear();
    P.sd_chunk.clear();
    for (int lg = 0; lg < kSd2Merge; ++lg) P.sd_span[lg] = 0;
    for (int p = 0; p <= SS_MAX_PLAYERS; ++p) P.sd_seg_off[p] = 0;
    P.strength.assign(static_cast<size_t>(np) * HS, 0u);
    if (need_sd) {
        if (nb != 5) {
            set_error("river showdowns need a 5-card board");
            return SS_ERR_INVALID;
        }
        struct C { uint32_t s; int a, b; };
        std::vector<C> combos;
        for (int a = 0; a < 52; ++a)
            for (int b = a + 1; b < 52; ++b)
                if (!on_board[a] && !on_board[b]) combos.push_back({rank7_host(board, a, b), a, b});
        std::stable_sort(combos.begin(), combos.end(),
                         [](const C &u, const C &v) { return u.s < v.s; });
        const int nc = static_cast<int>(combos.size());
        P.ncomb = nc;
        P.sd_combo.resize(nc);
        std::vector<int> pos_of(52 * 52, -1);
        std::vector<int> len(52, 0);
        for (int q = 0; q < nc; ++q) {
            pos_of[combos[q].a * 52 + combos[q].b] = q;
            pos_of[combos[q].b * 52 + combos[q].a] = q;
            P.sd_card_partner[combos[q].a * 52 + len[combos[q].a]] = static_cast<short>(combos[q].b);
            P.sd_card_list[combos[q].a * 52 + len[combos[q].a]++] = static_cast<short>(q);
            P.sd_card_partner[combos[q].b * 52 + len[combos[q].b]] = static_cast<short>(combos[q].a);
            P.sd_card_list[combos[q].b * 52 + len[combos[q].b]++] = static_cast<short>(q);
        }
        for (int q = 0; q < nc;) {
            int r = q;
            while (r < nc && combos[r].s == combos[q].s) ++r;
            for (int i = q; i < r; ++i) {
                P.sd_combo[i].lo = q;
                P.sd_combo[i].hi = r;
            }
            q = r;
        }
        auto count_below = [&](int card, int bound) {
            int c = 0;
            while (c < len[card] && P.sd_card_list[card * 52 + c] < bound) ++c;
            return static_cast<short>(c);
        };
        for (int q = 0; q < nc; ++q) {
            SdCombo &s = P.sd_combo[q];
            s.c1 = static_cast<short>(combos[q].a);
            s.c2 = static_cast<short>(combos[q].b);
            s.l1lo = count_below(combos[q].a, s.lo);
            s.l1hi = count_below(combos[q].a, s.hi);
            s.l2lo = count_below(combos[q].b, s.lo);
            s.l2hi = count_below(combos[q].b, s.hi);
        }
        for (int p = 0; p < np; ++p)
            for (int h = 0; h < P.H[p]; ++h) {
                const int a = pb.hands[p][2 * h], b = pb.hands[p][2 * h + 1];
                if (on_board[a] || on_board[b]) continue;
                const int q = pos_of[a * 52 + b];
                P.sd_pos[p * HS + h] = q;
                P.strength[p * HS + h] = combos[q].s;
            }
        for (int q = 0; q < nc; ++q) {
            P.sd_combo[q].d1 = static_cast<unsigned char>(dense[combos[q].a]);
            P.sd_combo[q].d2 = static_cast<unsigned char>(dense[combos[q].b]);
        }
        P.pos_hand.assign(static_cast<size_t>(np) * nc, -1);
        for (int p = 0; p < np; ++p)
            for (int h = 0; h < P.H[p]; ++h)
                if (P.sd_pos[p * HS + h] >= 0) P.pos_hand[static_cast<size_t>(p) * nc + P.sd_pos[p * HS + h]] = h;
        // per player: how many of its hands sit below each rank position
        P.pos_prefix.assign(static_cast<size_t>(np) * (nc + 1), 0);
        for (int p = 0; p < np; ++p)
            for (int q = 0; q < nc; ++q)
                P.pos_prefix[static_cast<size_t>(p) * (nc + 1) + q + 1] =
                    P.pos_prefix[static_cast<size_t>(p) * (nc + 1) + q] +
                    (P.pos_hand[static_cast<size_t>(p) * nc + q] >= 0 ? 1 : 0);
        P.sd_seg.clear();
        for (int p = 0; p < np; ++p) {
            P.sd_seg_off[p] = static_cast<int>(P.sd_seg.size() / 4);
            for (int q = 0; q < nc;) {
                const int hi = P.sd_combo[q].hi;
                bool has = false;
                for (int r = q; r < hi; ++r) has = has || P.pos_hand[static_cast<size_t>(p) * nc + r] >= 0;
                const size_t ns = P.sd_seg.size();
                const bool own = ns / 4 > static_cast<size_t>(P.sd_seg_off[p]);   // a segment of player p exists
                if (!has && own && P.sd_seg[ns - 2] == 0)
                    P.sd_seg[ns - 3] = hi;  // extend the previous run of groups without the player's hands
                else
                    P.sd_seg.insert(P.sd_seg.end(), {q, hi, has ? 1 : 0, 0});
                q = hi;
            }
        }
        P.sd_seg_off[np] = static_cast<int>(P.sd_seg.size() / 4);
        // runs of equal sweep cost: K = total cost / kSd2RunCost (1 .. kSd2Chunks,
        // and at most one wave of blocks over the traverser's three-way
        // showdowns), run k ends at the first segment boundary reaching k / K
        // of the cost
        P.sd_chunk.assign(static_cast<size_t>(np) * (kSd2Chunks + 1), 0);
        for (int p = 0; p < np; ++p) {
            const int a = P.sd_seg_off[p], b = P.sd_seg_off[p + 1];
            long long total = 0;
            for (int i = a; i < b; ++i) total += kSd2SegCost + P.sd_seg[4 * i + 1] - P.sd_seg[4 * i];
            const long long nt = static_cast<long long>(P.term[p][TK_SD2].size());
            const int K = static_cast<int>(std::max(
                1LL, std::min<long long>({kSd2Chunks, b - a, total / kSd2RunCost, nt ? kSd2Slots / nt : kSd2Chunks})));
            int *ch = P.sd_chunk.data() + static_cast<size_t>(p) * (kSd2Chunks + 1);
            ch[0] = a;
            long long acc = 0;
            int i = a;
            for (int k = 1; k <= kSd2Chunks; ++k) {
                if (k < K) {
                    const long long goal = total * k / K;
                    // at least one segment per run, and leave one for each later run
                    do {
                        acc += kSd2SegCost + P.sd_seg[4 * i + 1] - P.sd_seg[4 * i];
                        ++i;
                    } while (i < b - (K - k) && acc < goal);
                    ch[k] = i;
                } else {
                    ch[k] = b;
                }
            }
            for (int lg = 0; lg < kSd2Merge; ++lg)
                for (int r = 0; r < kSd2Chunks; r += 1 << lg) {
                    const int s0 = ch[r], s1 = ch[r + (1 << lg)];
                    if (s1 > s0)
                        P.sd_span[lg] = std::max(P.sd_span[lg], P.sd_seg[4 * (s1 - 1) + 1] - P.sd_seg[4 * s0]);
                }
        }
    }

    // per player: the range index of each dense-card pair (both orders), HS
    // where the range has no such hand (or it touches the board) -- the
    // two-opponent kernel keeps a zero after each staged reach row -- so it
    // gathers its combo matrices through this table without tests
    P.pair_idx.assign(static_cast<size_t>(np) * 52 * 52, P.HS);
    for (int p = 0; p < np; ++p)
        for (int h = 0; h < P.H[p]; ++h) {
            const int hc = P.hand_code[p * HS + h];
            if (hc & 0x10000) continue;
            const int a = (hc >> 20) & 63, b = (hc >> 26) & 63;
            P.pair_idx[(static_cast<size_t>(p) * 52 + a) * 52 + b] = h;
            P.pair_idx[(static_cast<size_t>(p) * 52 + b) * 52 + a] = h;
        }

    // per (traverser t, opponent o): the range index in o's range of each of
    // t's hands (the same two cards), HS where o has no such hand or the hand
    // touches the board -- the terminal kernels read an opponent's reach at the
    // traverser's own combo through it with one coalesced load per hand
    P.cross_idx.assign(static_cast<size_t>(np) * np * HS, P.HS);
    for (int t = 0; t < np; ++t)
        for (int o = 0; o < np; ++o)
            for (int h = 0; h < P.H[t]; ++h) {
                const int hc = P.hand_code[t * HS + h];
                if (hc & 0x10000) continue;
                const int a = (hc >> 20) & 63, b = (hc >> 26) & 63;
                P.cross_idx[(static_cast<size_t>(t) * np + o) * HS + h] =
                    P.pair_idx[(static_cast<size_t>(o) * 52 + a) * 52 + b];
            }

    double hsum = 0;
    for (int p = 0; p < np; ++p) hsum += P.H[p];
    P.node_hands = static_cast<double>(N) * hsum;
    // three-way showdowns: the run merge of this subgame's own launch
    for (int t = 0; t < np; ++t) {
        const int lg = sd2_merge_of(static_cast<int>(P.term[t][TK_SD2].size()));
        for (TermItem &it : P.term[t][TK_SD2]) it.kind_detail = lg;
    }
    return SS_OK;
}

}  // namespace ssb
