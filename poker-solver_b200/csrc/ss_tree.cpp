// ss_tree.cpp -- single-street N-player betting tree.
//
// Node ids, children order, leaf numbering and continuation expansion are part
// of the C ABI: callers index leaf_values by leaf_idx, frozen_action by node
// id and derive action labels from child bets.  The construction therefore
// follows the reference rules exactly (src/cuda/street_solve.cu:144-331 for
// the betting round, :336-460 for the continuation chains):
//   * a decision node gets its id before its subtrees, its children entries
//     after them;
//   * fold is offered only when facing a bet, then check/call, then one raise
//     per bet size (to_call + int(size * (pot + to_call)) when facing a bet,
//     int(size * pot) otherwise, clamped to the stack, one all-in at most),
//     then an explicit all-in if none of the sizes reached the stack, while
//     fewer than max_raises raises were made;
//   * the raise sets the actor's bet to (highest bet + amount) and adds the
//     amount to the pot, the stack never shrinks (both as in the reference);
//   * the round ends when every live player has acted and matched the
//     highest bet: showdown on the river, otherwise a leaf;
//   * each leaf becomes a chain of 4-way decisions, one per live player in
//     seat-index order, whose 4^n bottom nodes are the new leaves.
#include "ss_engine.h"

#include <cstring>
#include <vector>

namespace ssb {

namespace {

struct Street {
    int players;
    int max_raises;
    bool river;
    std::vector<int> order;
    std::vector<float> sizes;
    std::vector<int> board;
};

struct Seat {
    int bets[SS_MAX_PLAYERS];
    int acted[SS_MAX_PLAYERS];
    int live[SS_MAX_PLAYERS];
};

class Builder {
  public:
    explicit Builder(const Street &s) : st_(s) {}

    int grow(int seat_idx, int pot, int stack, const Seat &s, int raises);
    void expand_leaves();

    std::vector<SSNode> nodes;
    std::vector<int> kids;
    int leaves = 0;

  private:
    int make(int type) {
        SSNode n;
        std::memset(&n, 0, sizeof(n));
        n.type = type;
        n.player = -1;
        n.leaf_idx = -1;
        n.fold_player = -1;
        nodes.push_back(n);
        return static_cast<int>(nodes.size()) - 1;
    }
    void stamp(int id, int pot, const int *bets, const int *live) {
        SSNode &n = nodes[id];
        n.pot = pot;
        for (int i = 0; i < st_.players; ++i) n.bets[i] = bets[i];
        int nb = static_cast<int>(st_.board.size());
        for (int i = 0; i < nb && i < 5; ++i) n.board_cards[i] = st_.board[i];
        n.num_board = nb;
        n.num_players = 0;
        for (int i = 0; i < st_.players; ++i) {
            n.active_players[i] = live[i];
            n.num_players += live[i] ? 1 : 0;
        }
    }
    int next_live_seat(const int *live, int seat) const {
        for (int k = 1; k <= st_.players; ++k) {
            int s = (seat + k) % st_.players;
            int p = st_.order[s];
            if (p < st_.players && live[p]) return s;
        }
        return -1;
    }

    const Street &st_;
};

int Builder::grow(int seat, int pot, int stack, const Seat &s, int raises) {
    const int np = st_.players;
    int nlive = 0, top = 0;
    for (int i = 0; i < np; ++i) {
        if (!s.live[i]) continue;
        ++nlive;
        if (s.bets[i] > top) top = s.bets[i];
    }
    if (nlive <= 1) {
        int id = make(SS_NODE_FOLD);
        for (int i = 0; i < np; ++i)
            if (s.live[i]) { nodes[id].player = i; break; }
        stamp(id, pot, s.bets, s.live);
        return id;
    }
    bool settled = true;
    for (int i = 0; i < np && settled; ++i)
        if (s.live[i] && (!s.acted[i] || s.bets[i] != top)) settled = false;
    if (settled) {
        int id = make(st_.river ? SS_NODE_SHOWDOWN : SS_NODE_LEAF);
        if (!st_.river) nodes[id].leaf_idx = leaves++;
        stamp(id, pot, s.bets, s.live);
        return id;
    }
    const int actor = st_.order[seat];
    if (!s.live[actor]) {
        int nxt = next_live_seat(s.live, seat);
        if (nxt < 0) {
            int id = make(SS_NODE_SHOWDOWN);
            stamp(id, pot, s.bets, s.live);
            return id;
        }
        return grow(nxt, pot, stack, s, raises);
    }

    const int me = make(SS_NODE_DECISION);
    nodes[me].player = actor;
    stamp(me, pot, s.bets, s.live);

    int to_call = top - s.bets[actor];
    if (to_call < 0) to_call = 0;
    int nxt = next_live_seat(s.live, seat);
    if (nxt < 0) nxt = seat;

    int out[16];
    int n_out = 0;
    if (to_call > 0) {
        Seat f = s;
        f.live[actor] = 0;
        out[n_out++] = grow(nxt, pot, stack, f, raises);
    }
    {
        Seat c = s;
        c.bets[actor] = top;
        c.acted[actor] = 1;
        out[n_out++] = grow(nxt, pot + to_call, stack, c, raises);
    }
    auto raise_to = [&](int amount) {
        Seat r = s;
        r.bets[actor] = top + amount;
        r.acted[actor] = 1;
        for (int p = 0; p < np; ++p)
            if (p != actor && s.live[p]) r.acted[p] = 0;
        out[n_out++] = grow(nxt, pot + amount, stack, r, raises + 1);
    };
    if (raises < st_.max_raises && n_out < 14) {
        bool allin = false;
        for (size_t i = 0; i < st_.sizes.size() && n_out < 14; ++i) {
            const float f = st_.sizes[i];
            int amount = to_call == 0 ? static_cast<int>(f * static_cast<float>(pot))
                                      : to_call + static_cast<int>(f * static_cast<float>(pot + to_call));
            if (amount >= stack) amount = stack;
            if (amount <= to_call) continue;
            if (amount >= stack) {
                if (allin) continue;
                allin = true;
            }
            raise_to(amount);
        }
        if (!allin && stack > to_call && n_out < 14) raise_to(stack);
    }
    const int at = static_cast<int>(kids.size());
    kids.insert(kids.end(), out, out + n_out);
    nodes[me].first_child = at;
    nodes[me].num_children = n_out;
    return me;
}

void Builder::expand_leaves() {
    std::vector<int> old;
    for (size_t i = 0; i < nodes.size(); ++i)
        if (nodes[i].type == SS_NODE_LEAF) old.push_back(static_cast<int>(i));
    leaves = 0;
    for (int id : old) {
        const SSNode base = nodes[id];
        int chain[SS_MAX_PLAYERS], len = 0;
        for (int p = 0; p < st_.players; ++p)
            if (base.active_players[p]) chain[len++] = p;
        if (len == 0) continue;
        nodes[id].type = SS_NODE_DECISION;
        nodes[id].player = chain[0];
        nodes[id].leaf_idx = -1;
        std::vector<int> layer(1, id), below;
        for (int step = 0; step < len; ++step) {
            const bool bottom = step == len - 1;
            below.clear();
            for (int parent : layer) {
                if (step > 0) {
                    nodes[parent].type = SS_NODE_DECISION;
                    nodes[parent].player = chain[step];
                }
                int made[SS_NUM_CONT_STRATS];
                for (int k = 0; k < SS_NUM_CONT_STRATS; ++k) {
                    int x = make(bottom ? SS_NODE_LEAF : SS_NODE_DECISION);
                    SSNode &n = nodes[x];
                    if (bottom) n.leaf_idx = leaves++;
                    n.pot = base.pot;
                    std::memcpy(n.bets, base.bets, sizeof(n.bets));
                    for (int i = 0; i < base.num_board && i < 5; ++i) n.board_cards[i] = base.board_cards[i];
                    n.num_board = base.num_board;
                    n.num_players = 0;
                    for (int i = 0; i < st_.players; ++i) {
                        n.active_players[i] = base.active_players[i];
                        n.num_players += base.active_players[i] ? 1 : 0;
                    }
                    made[k] = x;
                    if (!bottom) below.push_back(x);
                }
                const int at = static_cast<int>(kids.size());
                kids.insert(kids.end(), made, made + SS_NUM_CONT_STRATS);
                nodes[parent].first_child = at;
                nodes[parent].num_children = SS_NUM_CONT_STRATS;
            }
            layer.swap(below);
        }
    }
}

}  // namespace

int build_street_tree(const int *board, int num_board, int starting_pot, int effective_stack,
                      const float *bet_sizes, int num_bet_sizes, int num_players,
                      const int *acting_order, int is_river, int use_cont_strats, int max_raises,
                      BuiltTree *out) {
    if (num_players < 1 || num_players > SS_MAX_PLAYERS || !acting_order) {
        set_error("ss_build_tree: num_players must be 1..6 with an acting order");
        return SS_ERR_INVALID;
    }
    if (num_board < 0 || num_board > SS_MAX_BOARD || (num_board > 0 && !board) ||
        num_bet_sizes < 0 || (num_bet_sizes > 0 && !bet_sizes) || max_raises < 0) {
        set_error("ss_build_tree: bad board, bet sizes or raise cap");
        return SS_ERR_INVALID;
    }
    for (int i = 0; i < num_players; ++i)
        if (acting_order[i] < 0 || acting_order[i] >= num_players) {
            set_error("ss_build_tree: acting_order entries must be player indices");
            return SS_ERR_INVALID;
        }
    Street st;
    st.players = num_players;
    st.max_raises = max_raises;
    st.river = is_river != 0;
    st.order.assign(acting_order, acting_order + num_players);
    st.sizes.assign(bet_sizes, bet_sizes + num_bet_sizes);
    st.board.assign(board, board + num_board);

    Builder b(st);
    Seat s;
    std::memset(&s, 0, sizeof(s));
    for (int i = 0; i < num_players; ++i) s.live[i] = 1;
    b.grow(0, starting_pot, effective_stack, s, 0);
    if (use_cont_strats && !is_river && b.leaves > 0) b.expand_leaves();

    out->nodes.swap(b.nodes);
    out->children.swap(b.kids);
    out->num_leaves = b.leaves;

    // breadth-first order and depth from node 0 (street_solve.cu:1238-1259)
    const int n = static_cast<int>(out->nodes.size());
    out->level_order.assign(n, 0);
    out->node_depth.assign(n, 0);
    out->max_depth = 0;
    int head = 0, tail = 0;
    out->level_order[tail++] = 0;
    while (head < tail) {
        const int x = out->level_order[head++];
        const int d = out->node_depth[x];
        if (d > out->max_depth) out->max_depth = d;
        const SSNode &nd = out->nodes[x];
        for (int a = 0; a < nd.num_children; ++a) {
            const int c = out->children[nd.first_child + a];
            out->node_depth[c] = d + 1;
            out->level_order[tail++] = c;
        }
    }
    return SS_OK;
}

}  // namespace ssb
