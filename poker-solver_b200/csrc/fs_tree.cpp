// fs_tree.cpp -- the flop-through-river betting tree (fs_build_tree).
//
// Node numbering, children order and the node fields are part of the ABI
// (callers index strategies by node id and find the turn roots by walking the
// flop-ending chance nodes), so the construction follows the reference's
// rules (flop_solve.cu:72-362, 894-972), written independently:
//   * two players, player 0 acts first on every street; one raise per street;
//   * a street ends when both have acted with equal bets: a showdown on the
//     river, else a chance node that deals the next card;
//   * fold only when facing a bet; check or call (the second action's call
//     ends the street); a bet or raise of to_call + int(f * (pot + to_call))
//     (int(f * pot) unopened), capped at the stack; a capped bet becomes an
//     all-in node (the opponent folds or calls, the call ends the street) --
//     at most one, and an explicit one is added when no size reached the
//     stack and fewer than seven actions exist;
//   * a node is numbered when it is created, before its subtrees; a node's
//     children slots are reserved after its subtrees are built;
//   * the flop street uses the caller's bet sizes; then every chance node
//     without children (in node order, those existing before the pass) gets
//     one turn subtree per undealt card with a single 0.75-pot size, and the
//     same again for the river; those subtrees start with pot = the chance
//     node's pot, no bets, and a stack of 10000 minus player 0's bet at the
//     chance node (the reference's fixed figure, kept since it shapes the
//     tree).
#include "fs_engine.h"

#include <cstdlib>
#include <cstring>
#include <vector>

namespace ssb {
namespace fs {

namespace {

constexpr int kRaiseCap = 1;       // flop_solve.cu:25
constexpr float kLaterSize = 0.75f;
constexpr int kLaterStack = 10000;

class Builder {
  public:
    std::vector<FSNode> nodes;
    std::vector<int> kids;

    int make(int type, int player, int pot, int b0, int b1, const int *board, int nb) {
        FSNode n;
        std::memset(&n, 0, sizeof(n));
        n.type = type;
        n.player = player;
        n.pot = pot;
        n.bets[0] = b0;
        n.bets[1] = b1;
        for (int i = 0; i < nb; ++i) n.board_cards[i] = board[i];
        n.num_board = nb;
        nodes.push_back(n);
        return static_cast<int>(nodes.size()) - 1;
    }

    void attach(int node, const int *c, int count) {
        const int at = static_cast<int>(kids.size());
        kids.insert(kids.end(), c, c + count);
        nodes[node].first_child = at;
        nodes[node].num_children = count;
    }

    // the node that closes a street: showdown on the river, else a chance node
    int close(bool river, int pot, int b0, int b1, const int *board, int nb) {
        return make(river ? FS_NODE_SHOWDOWN : FS_NODE_CHANCE, -1, pot, b0, b1, board, nb);
    }

    // an all-in of `actor` for `amount` more chips: the opponent folds or calls
    int all_in(bool river, int actor, int pot, int b0, int b1, int to_call, int amount, const int *board, int nb) {
        int n0 = b0, n1 = b1;
        (actor == 0 ? n0 : n1) += amount;
        const int pot2 = pot + amount;
        const int ai = make(FS_NODE_DECISION, 1 - actor, pot2, n0, n1, board, nb);
        const int fold = make(FS_NODE_FOLD, actor, pot2, n0, n1, board, nb);
        // the call matches the all-in bet
        const int c0 = actor == 0 ? n0 : n1, c1 = actor == 0 ? n0 : n1;
        const int call = close(river, pot2 + (amount - to_call), actor == 0 ? n0 : c0, actor == 0 ? c1 : n1, board, nb);
        const int ch[2] = {fold, call};
        attach(ai, ch, 2);
        return ai;
    }

    int street(bool river, int player, int pot, int stack, int b0, int b1, int raises, int acted,
               const float *sizes, int ns, const int *board, int nb) {
        const int to_call = std::max(0, player == 0 ? b1 - b0 : b0 - b1);
        if (acted >= 2 && b0 == b1) return close(river, pot, b0, b1, board, nb);
        const int node = make(FS_NODE_DECISION, player, pot, b0, b1, board, nb);
        int ch[8], nc = 0;
        if (to_call > 0) ch[nc++] = make(FS_NODE_FOLD, 1 - player, pot, b0, b1, board, nb);
        if (to_call == 0) {
            ch[nc++] = street(river, 1 - player, pot, stack, b0, b1, raises, acted + 1, sizes, ns, board, nb);
        } else {
            const int m = player == 0 ? b1 : b0;   // the call matches the opponent's bet
            const int c0 = player == 0 ? m : b0, c1 = player == 0 ? b1 : m;
            if (acted >= 1)
                ch[nc++] = close(river, pot + to_call, c0, c1, board, nb);
            else
                ch[nc++] = street(river, 1 - player, pot + to_call, stack - to_call, c0, c1, raises, acted + 1, sizes,
                                  ns, board, nb);
        }
        if (raises < kRaiseCap) {
            bool shoved = false;
            for (int i = 0; i < ns; ++i) {
                int amount = to_call == 0 ? static_cast<int>(sizes[i] * pot)
                                          : to_call + static_cast<int>(sizes[i] * (pot + to_call));
                if (amount >= stack) amount = stack;
                if (amount <= to_call) continue;
                if (amount >= stack) {
                    if (shoved) continue;
                    shoved = true;
                    ch[nc++] = all_in(river, player, pot, b0, b1, to_call, amount, board, nb);
                } else {
                    int n0 = b0, n1 = b1;
                    (player == 0 ? n0 : n1) += amount;
                    ch[nc++] = street(river, 1 - player, pot + amount, stack - amount + to_call, n0, n1, raises + 1,
                                      acted + 1, sizes, ns, board, nb);
                }
            }
            if (!shoved && stack > to_call && nc < 7)
                ch[nc++] = all_in(river, player, pot, b0, b1, to_call, stack, board, nb);
        }
        attach(node, ch, nc);
        return node;
    }

    // one child subtree per undealt card under every childless chance node
    // that exists now, in node order
    void deal(float size) {
        std::vector<int> todo;
        for (int i = 0; i < static_cast<int>(nodes.size()); ++i) {
            const FSNode &n = nodes[i];
            if (n.type == FS_NODE_CHANCE && n.num_board < 5 && n.num_children == 0) todo.push_back(i);
        }
        for (int x : todo) {
            const FSNode snap = nodes[x];   // copied: subtrees append to `nodes`
            bool used[52] = {};
            for (int b = 0; b < snap.num_board; ++b) used[snap.board_cards[b]] = true;
            int cards[52], ncard = 0;
            for (int c = 0; c < 52; ++c)
                if (!used[c]) cards[ncard++] = c;
            const int at = static_cast<int>(kids.size());
            kids.resize(kids.size() + ncard);
            nodes[x].first_child = at;
            nodes[x].num_children = ncard;
            const bool river = snap.num_board + 1 == 5;
            const int stack = std::max(0, kLaterStack - snap.bets[0]);
            for (int k = 0; k < ncard; ++k) {
                int board[5];
                for (int b = 0; b < snap.num_board; ++b) board[b] = snap.board_cards[b];
                board[snap.num_board] = cards[k];
                const float s = size;
                kids[at + k] = street(river, 0, snap.pot, stack, 0, 0, 0, 0, &s, 1, board, snap.num_board + 1);
            }
        }
    }
};

template <class T>
T *copy_out(const std::vector<T> &v) {
    T *p = static_cast<T *>(std::malloc(std::max<size_t>(v.size(), 1) * sizeof(T)));
    if (p && !v.empty()) std::memcpy(p, v.data(), v.size() * sizeof(T));
    return p;
}

}  // namespace

int build_tree(const int *flop, int starting_pot, int effective_stack, const float *sizes, int num_sizes,
               FSTreeData *out) {
    std::memset(out, 0, sizeof(*out));
    if (!flop || (num_sizes > 0 && !sizes) || num_sizes < 0) {
        set_error("fs_build_tree: missing board or bet sizes");
        return SS_ERR_INVALID;
    }
    bool seen[52] = {};
    for (int i = 0; i < 3; ++i) {
        if (flop[i] < 0 || flop[i] > 51 || seen[flop[i]]) {
            set_error("fs_build_tree: the flop must be three distinct cards 0..51");
            return SS_ERR_INVALID;
        }
        seen[flop[i]] = true;
    }
    Builder b;
    b.street(false, 0, starting_pot, effective_stack, 0, 0, 0, 0, sizes, num_sizes, flop, 3);
    b.deal(kLaterSize);   // turn
    b.deal(kLaterSize);   // river
    const int N = static_cast<int>(b.nodes.size());
    // breadth-first order and depths
    std::vector<int> order, depth(N, 0);
    order.reserve(N);
    order.push_back(0);
    int max_depth = 0;
    for (size_t q = 0; q < order.size(); ++q) {
        const FSNode &n = b.nodes[order[q]];
        max_depth = std::max(max_depth, depth[order[q]]);
        for (int a = 0; a < n.num_children; ++a) {
            const int c = b.kids[n.first_child + a];
            depth[c] = depth[order[q]] + 1;
            order.push_back(c);
        }
    }
    std::vector<int> dec, sd;
    for (int i = 0; i < N; ++i) {
        if (b.nodes[i].type == FS_NODE_DECISION) dec.push_back(i);
        if (b.nodes[i].type == FS_NODE_SHOWDOWN) sd.push_back(i);
    }
    out->nodes = copy_out(b.nodes);
    out->children = copy_out(b.kids);
    out->level_order = copy_out(order);
    out->node_depth = copy_out(depth);
    out->decision_node_indices = copy_out(dec);
    out->showdown_node_indices = copy_out(sd);
    if (!out->nodes || !out->children || !out->level_order || !out->node_depth || !out->decision_node_indices ||
        !out->showdown_node_indices) {
        free_tree(out);
        set_error("fs_build_tree: out of host memory");
        return SS_ERR_NOMEM;
    }
    out->num_nodes = N;
    out->num_children_total = static_cast<int>(b.kids.size());
    out->max_depth = max_depth;
    out->num_decision_nodes = static_cast<int>(dec.size());
    out->num_showdown_nodes = static_cast<int>(sd.size());
    return SS_OK;
}

void free_tree(FSTreeData *t) {
    if (!t) return;
    std::free(t->nodes);
    std::free(t->children);
    std::free(t->level_order);
    std::free(t->node_depth);
    std::free(t->decision_node_indices);
    std::free(t->showdown_node_indices);
    std::memset(t, 0, sizeof(*t));
}

}  // namespace fs
}  // namespace ssb
