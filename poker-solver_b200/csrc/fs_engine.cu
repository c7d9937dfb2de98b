// fs_engine.cu -- the multi-street two-player solver on the GPU.
//
// The reference (flop_solve.cu:974-1270) keeps reach and values per node for
// every hand, re-runs regret matching over all decision nodes and
// re-propagates the opponent's reach through every level for each traverser,
// and launches one kernel per tree level and kind with a host sync per
// iteration.  Here the street solver's machinery carries over:
//   * reach is stored per sequence (one row per decision edge): a chance node
//     deals a card but changes no player's reach, so it is transparent, and a
//     player's reach is re-propagated once per iteration, after its own
//     regret update (k_reach, regret matching fused in);
//   * values are written only for terminals and the traverser's decision
//     nodes; an edge's value is the sum of its frontier rows -- through the
//     opponent's decisions and through chance nodes, whose average becomes a
//     weight 1 / cards dealt folded into each frontier row when it is written
//     (the items' `scale`), so k_cfv sums rows unchanged;
//   * terminals: one block per terminal stages the opponent's reach row,
//     cards and (showdowns) 7-card strengths for the node's board in shared
//     memory; each thread sums its traverser hands over them (at most 200
//     hands per player by the ABI: 40 K operations per terminal);
//   * strengths: once per solve for every river board of the tree with the
//     device ranker (ss_rank.cuh), instead of once per showdown node;
//   * iterations are captured as CUDA graphs with the counter on the device.
// fs_solve_gpu_extract_all reads the average strategy of every node and the
// last traverser's values at every node (terminals, both players' decisions,
// chance averages) from the same solve: the strategy of the last pass is kept
// for the read-out.
#include "fs_engine.h"
#include "ss_kernels.h"
#include "ss_rank.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <string>

namespace ssb {
namespace fs {

// ---------------------------------------------------------------------------
// planner
// ---------------------------------------------------------------------------

namespace {

bool fail(const std::string &m) {
    set_error("fs: " + m);
    return false;
}

bool validate(const FSTreeData &td, FsPlan &P) {
    if (!td.nodes || !td.children || td.num_nodes < 1) return fail("tree has no nodes");
    for (int p = 0; p < 2; ++p) {
        if (td.num_hands[p] < 0 || td.num_hands[p] > FS_MAX_HANDS) return fail("num_hands must be 0..200");
        P.H[p] = td.num_hands[p];
        for (int h = 0; h < P.H[p]; ++h) {
            const int a = td.hands[p][h][0], b = td.hands[p][h][1];
            if (a < 0 || a > 51 || b < 0 || b > 51 || a == b) return fail("hands must be two distinct cards 0..51");
        }
    }
    P.max_h = std::max(P.H[0], P.H[1]);
    if (P.max_h == 0) return fail("both ranges are empty");
    for (int i = 0; i < td.num_nodes; ++i) {
        const FSNode &n = td.nodes[i];
        if (n.num_board < 3 || n.num_board > 5) return fail("node board must hold 3..5 cards");
        if (n.type == FS_NODE_DECISION || n.type == FS_NODE_CHANCE) {
            if (n.num_children < 1 || n.first_child < 0 || n.first_child + n.num_children > td.num_children_total)
                return fail("node " + std::to_string(i) + " has bad children");
            if (n.type == FS_NODE_DECISION && (n.num_children > FS_MAX_ACTIONS || n.player < 0 || n.player > 1))
                return fail("decision node " + std::to_string(i) + " needs a player and 1..6 actions");
            for (int a = 0; a < n.num_children; ++a) {
                const int c = td.children[n.first_child + a];
                if (c <= 0 || c >= td.num_nodes) return fail("child id out of range");
            }
        } else if (n.type == FS_NODE_FOLD) {
            if (n.player < 0 || n.player > 1 || n.num_children != 0) return fail("fold node without a winner");
        } else if (n.type == FS_NODE_SHOWDOWN) {
            if (n.num_board != 5 || n.num_children != 0) return fail("showdown before the river");
        } else {
            return fail("unknown node type");
        }
        for (int b = 0; b < n.num_board; ++b)
            if (n.board_cards[b] < 0 || n.board_cards[b] > 51) return fail("board card out of range");
    }
    if (td.nodes[0].type != FS_NODE_DECISION) return fail("node 0 must be a decision node");
    return true;
}

}  // namespace

int build_plan(const FSTreeData &td, FsPlan *out) {
    FsPlan &P = *out;
    if (!validate(td, P)) return SS_ERR_INVALID;
    const int N = td.num_nodes;
    P.N = N;
    P.HS = (P.max_h + 31) / 32 * 32;
    const FSNode *nd = td.nodes;
    auto child = [&](int x, int a) { return td.children[nd[x].first_child + a]; };
    // breadth-first order; every node reached once
    std::vector<int> order{0}, parent(N, -2), pact(N, -1), depth(N, 0);
    parent[0] = -1;
    for (size_t q = 0; q < order.size(); ++q) {
        const int x = order[q];
        if (nd[x].type != FS_NODE_DECISION && nd[x].type != FS_NODE_CHANCE) continue;
        for (int a = 0; a < nd[x].num_children; ++a) {
            const int c = child(x, a);
            if (parent[c] != -2) {
                set_error("fs: node " + std::to_string(c) + " is reached twice: not a tree");
                return SS_ERR_INVALID;
            }
            parent[c] = x;
            pact[c] = a;
            depth[c] = depth[x] + 1;
            order.push_back(c);
        }
    }
    if (static_cast<int>(order.size()) != N) {
        set_error("fs: some nodes are not reachable from node 0");
        return SS_ERR_INVALID;
    }
    P.root_player = nd[0].player;
    P.root_na = nd[0].num_children;
    P.first_edge.assign(N, -1);
    P.edge_node.clear();
    for (int x : order)
        if (nd[x].type == FS_NODE_DECISION) {
            P.first_edge[x] = static_cast<int>(P.edge_node.size());
            for (int a = 0; a < nd[x].num_children; ++a) P.edge_node.push_back(x);
        }
    P.E = static_cast<int>(P.edge_node.size());
    const int E = P.E;
    for (int i = 0; i < N; ++i)
        if (nd[i].type == FS_NODE_DECISION) P.dec_nodes.push_back(i);
    // each player's sequence (reach row) and own-decision depth at every node
    std::vector<int> last(2 * static_cast<size_t>(N)), pdepth(2 * static_cast<size_t>(N), 0);
    for (int x : order)
        for (int p = 0; p < 2; ++p) {
            if (x == 0) {
                last[p] = E + p;
                continue;
            }
            const int par = parent[x];
            const bool acted = nd[par].type == FS_NODE_DECISION && nd[par].player == p;
            last[2 * x + p] = acted ? P.first_edge[par] + pact[x] : last[2 * par + p];
            pdepth[2 * x + p] = pdepth[2 * par + p] + (acted ? 1 : 0);
        }
    for (int p = 0; p < 2; ++p)
        for (int x : order) {
            if (nd[x].type != FS_NODE_DECISION || nd[x].player != p) continue;
            const int lev = pdepth[2 * x + p];
            if (static_cast<int>(P.reach_levels[p].size()) <= lev) P.reach_levels[p].resize(lev + 1);
            ReachItem it;
            it.first_edge = P.first_edge[x];
            it.na = nd[x].num_children;
            it.parent_row = last[2 * x + p];
            it.frozen = -1;
            P.reach_levels[p][lev].push_back(it);
        }
    // frontiers: through the other player's decisions and through chance nodes
    P.fr_off.assign(E + 1, 0);
    std::vector<int> stack;
    for (int e = 0; e < E; ++e) {
        const int x = P.edge_node[e], p = nd[x].player;
        stack.assign(1, child(x, e - P.first_edge[x]));
        while (!stack.empty()) {
            const int y = stack.back();
            stack.pop_back();
            const bool pass = nd[y].type == FS_NODE_CHANCE || (nd[y].type == FS_NODE_DECISION && nd[y].player != p);
            if (!pass) {
                P.fr_items.push_back(y);
                continue;
            }
            for (int a = nd[y].num_children - 1; a >= 0; --a) stack.push_back(child(y, a));
        }
        P.fr_off[e + 1] = static_cast<int>(P.fr_items.size());
    }
    // per traverser: the chance weight of every node within its frontier
    // (1 below a traverser decision, divided by the cards at each chance node)
    std::vector<double> w(N);
    for (int t = 0; t < 2; ++t) {
        for (int x : order) {
            if (x == 0) {
                w[x] = 1.0;
                continue;
            }
            const int par = parent[x];
            w[x] = nd[par].type == FS_NODE_DECISION && nd[par].player == t ? 1.0
                   : nd[par].type == FS_NODE_CHANCE ? w[par] / nd[par].num_children
                                                    : w[par];
        }
        // value / regret levels: height in own decisions, bottom-up
        std::vector<int> height(N, 0);
        P.cfv_levels[t].clear();
        for (int q = N - 1; q >= 0; --q) {
            const int x = order[q];
            if (nd[x].type != FS_NODE_DECISION || nd[x].player != t) continue;
            int h = 0;
            const int fe = P.first_edge[x];
            for (int k = P.fr_off[fe]; k < P.fr_off[fe + nd[x].num_children]; ++k) {
                const int y = P.fr_items[k];
                if (nd[y].type == FS_NODE_DECISION) h = std::max(h, height[y] + 1);
            }
            height[x] = h;
            if (static_cast<int>(P.cfv_levels[t].size()) <= h) P.cfv_levels[t].resize(h + 1);
            CfvItem it;
            it.first_edge = fe;
            it.na = nd[x].num_children;
            it.frozen = -1;
            it.node = x;
            it.scale = static_cast<float>(w[x]);
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
    // river boards of the showdowns, and the terminal items
    const float half_start = static_cast<float>(nd[0].pot) * 0.5f;   // flop_solve.cu:755
    std::vector<int> board_row(N, -1);
    {
        std::vector<long long> keys;
        for (int x = 0; x < N; ++x)
            if (nd[x].type == FS_NODE_SHOWDOWN) {
                long long k = 0;
                for (int b = 0; b < 5; ++b) k = k * 64 + nd[x].board_cards[b];
                keys.push_back(k);
            }
        std::vector<long long> uk = keys;
        std::sort(uk.begin(), uk.end());
        uk.erase(std::unique(uk.begin(), uk.end()), uk.end());
        for (long long k : uk)   // card b is base-64 digit 4 - b
            for (int b = 0; b < 5; ++b) P.sboards.push_back(static_cast<int>((k >> (6 * (4 - b))) & 63));
        for (int x = 0; x < N; ++x)
            if (nd[x].type == FS_NODE_SHOWDOWN) {
                long long k = 0;
                for (int b = 0; b < 5; ++b) k = k * 64 + nd[x].board_cards[b];
                board_row[x] = static_cast<int>(std::lower_bound(uk.begin(), uk.end(), k) - uk.begin());
            }
    }
    for (int t = 0; t < 2; ++t) {
        // chance weights for traverser t again (the loop above kept t = 1's)
        for (int x : order) {
            if (x == 0) {
                w[x] = 1.0;
                continue;
            }
            const int par = parent[x];
            w[x] = nd[par].type == FS_NODE_DECISION && nd[par].player == t ? 1.0
                   : nd[par].type == FS_NODE_CHANCE ? w[par] / nd[par].num_children
                                                    : w[par];
        }
        P.term[t].clear();
        for (int x = 0; x < N; ++x) {
            const FSNode &n = nd[x];
            if (n.type != FS_NODE_FOLD && n.type != FS_NODE_SHOWDOWN) continue;
            FsTermItem it;
            std::memset(&it, 0, sizeof(it));
            it.node = x;
            it.kind = n.type == FS_NODE_FOLD ? 0 : 1;
            it.opp_row = last[2 * x + (1 - t)];
            it.sboard = board_row[x];
            if (n.type == FS_NODE_FOLD) {
                const int winner = n.player, loser = 1 - winner;
                it.payoff = t == winner ? half_start + static_cast<float>(n.bets[loser])
                                        : -(half_start + static_cast<float>(n.bets[t]));
            }
            it.half_pot = static_cast<float>(n.pot) * 0.5f;
            it.scale = static_cast<float>(w[x]);
            it.nb = n.num_board;
            for (int b = 0; b < n.num_board; ++b) it.board[b] = n.board_cards[b];
            P.term[t].push_back(it);
        }
        // folds first, then showdowns (one launch each)
        std::stable_partition(P.term[t].begin(), P.term[t].end(), [](const FsTermItem &i) { return i.kind == 0; });
        P.nfold[t] = static_cast<int>(std::count_if(P.term[t].begin(), P.term[t].end(),
                                                    [](const FsTermItem &i) { return i.kind == 0; }));
    }
    // hands, and per player the hands holding each card (folds)
    const int HSi = P.HS;
    P.hand_cards.assign(2 * static_cast<size_t>(HSi), -1);
    for (int p = 0; p < 2; ++p)
        for (int h = 0; h < P.H[p]; ++h) P.hand_cards[p * HSi + h] = td.hands[p][h][0] | (td.hands[p][h][1] << 8);
    P.f_coff.assign(2 * 53, 0);
    P.f_clist.assign(2 * 2 * static_cast<size_t>(HSi), 0);
    for (int p = 0; p < 2; ++p) {
        std::vector<std::vector<int>> byc(52);
        for (int h = 0; h < P.H[p]; ++h) {
            byc[td.hands[p][h][0]].push_back(h);
            byc[td.hands[p][h][1]].push_back(h);
        }
        int at = 0;
        for (int c = 0; c < 52; ++c) {
            P.f_coff[p * 53 + c] = at;
            for (int h : byc[c]) P.f_clist[p * 2 * HSi + at++] = h;
        }
        P.f_coff[p * 53 + 52] = at;
    }
    // showdown tables per river board (see fs_engine.h)
    const int nsb = static_cast<int>(P.sboards.size() / 5);
    P.sd_str.assign(static_cast<size_t>(nsb) * 2 * HSi, 0u);
    P.sd_ord.assign(static_cast<size_t>(nsb) * 2 * HSi, -1);
    P.sd_hpos.assign(static_cast<size_t>(nsb) * 2 * HSi * 4, 0);
    P.sd_coff.assign(static_cast<size_t>(nsb) * 2 * 53, 0);
    P.sd_clist.assign(static_cast<size_t>(nsb) * 2 * 2 * HSi, 0);
    for (int bi = 0; bi < nsb; ++bi) {
        const int *bd = &P.sboards[5 * bi];
        std::vector<unsigned> srt[2];
        for (int p = 0; p < 2; ++p) {
            unsigned *str = &P.sd_str[(static_cast<size_t>(bi) * 2 + p) * HSi];
            for (int h = 0; h < P.H[p]; ++h) str[h] = rank7_host(bd, td.hands[p][h][0], td.hands[p][h][1]);
            int *ord = &P.sd_ord[(static_cast<size_t>(bi) * 2 + p) * HSi];
            std::vector<int> idx(P.H[p]);
            for (int h = 0; h < P.H[p]; ++h) idx[h] = h;
            std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) { return str[x] < str[y]; });
            std::vector<int> pos(P.H[p]);
            for (int k = 0; k < P.H[p]; ++k) {
                ord[k] = idx[k];
                pos[idx[k]] = k;
                srt[p].push_back(str[idx[k]]);
            }
            // card lists of this player as the opponent, by position
            std::vector<std::vector<int>> byc(52);
            for (int k = 0; k < P.H[p]; ++k) {
                byc[td.hands[p][idx[k]][0]].push_back(k);
                byc[td.hands[p][idx[k]][1]].push_back(k);
            }
            int *coff = &P.sd_coff[(static_cast<size_t>(bi) * 2 + p) * 53];
            int *cl = &P.sd_clist[(static_cast<size_t>(bi) * 2 + p) * 2 * HSi];
            int at = 0;
            for (int c = 0; c < 52; ++c) {
                coff[c] = at;
                for (int k : byc[c]) cl[at++] = k;
            }
            coff[52] = at;
        }
        for (int t = 0; t < 2; ++t) {
            const int o = 1 - t;
            const unsigned *st = &P.sd_str[(static_cast<size_t>(bi) * 2 + t) * HSi];
            const unsigned *so = &P.sd_str[(static_cast<size_t>(bi) * 2 + o) * HSi];
            const int *coff = &P.sd_coff[(static_cast<size_t>(bi) * 2 + o) * 53];
            const int *cl = &P.sd_clist[(static_cast<size_t>(bi) * 2 + o) * 2 * HSi];
            const int *ordo = &P.sd_ord[(static_cast<size_t>(bi) * 2 + o) * HSi];
            for (int h = 0; h < P.H[t]; ++h) {
                const unsigned s = st[h];
                const int lo = static_cast<int>(std::lower_bound(srt[o].begin(), srt[o].end(), s) - srt[o].begin());
                const int hi = static_cast<int>(std::upper_bound(srt[o].begin(), srt[o].end(), s) - srt[o].begin());
                const int c1 = td.hands[t][h][0], c2 = td.hands[t][h][1];
                int cnt[2][2];
                const int cs[2] = {c1, c2};
                for (int j = 0; j < 2; ++j) {
                    int below = 0, upto = 0;
                    for (int k = coff[cs[j]]; k < coff[cs[j] + 1]; ++k) {
                        const unsigned x = so[ordo[cl[k]]];
                        below += x < s;
                        upto += x <= s;
                    }
                    cnt[j][0] = below;
                    cnt[j][1] = upto;
                }
                int *hp = &P.sd_hpos[((static_cast<size_t>(bi) * 2 + t) * HSi + h) * 4];
                hp[0] = lo | (hi << 16);
                hp[1] = c1 | (c2 << 8);
                hp[2] = cnt[0][0] | (cnt[0][1] << 16);
                hp[3] = cnt[1][0] | (cnt[1][1] << 16);
            }
        }
    }
    // read-out levels: BFS depth, deepest first
    int maxd = 0;
    for (int x = 0; x < N; ++x) maxd = std::max(maxd, depth[x]);
    P.depth_off.assign(maxd + 2, 0);
    std::vector<std::vector<int>> byd(maxd + 1);
    for (int x : order) byd[depth[x]].push_back(x);
    for (int d = maxd; d >= 0; --d) {
        P.depth_nodes.insert(P.depth_nodes.end(), byd[d].begin(), byd[d].end());
        P.depth_off[maxd - d + 1] = static_cast<int>(P.depth_nodes.size());
    }
    return SS_OK;
}

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------

namespace {

constexpr int kFsThreads = 256;

// Folds (flop_solve.cu:731-779): payoff x the opponent's reach over hands
// sharing no card with the traverser's hand {a, b} or with the node's board.
// One block per terminal: the opponent's hands the board leaves are staged
// (reach in FP64, and whether it is positive); per card c their sums u(c),
// and F in all; then per traverser hand
//   mass = F - u(a) - u(b) + (the opponent's reach on the combo {a, b}),
// the last term from the opponent's list of card a.  The same sums over 0/1
// count the opponent hands with positive reach; none gives exactly 0, as the
// reference's sum of zeros does.
struct FsTables {
    const int *hand_cards;                    // [2][HS]
    const int *f_coff, *f_clist;              // [2][53], [2][2 HS]
    const unsigned *sd_str;                   // [nsb][2][HS]
    const int *sd_ord, *sd_hpos, *sd_coff, *sd_clist;
    int HS, H0, H1;
};

__global__ void __launch_bounds__(kFsThreads) k_fs_fold(const FsTermItem *__restrict__ items, int trav,
                                                       const float *__restrict__ reach, FsTables T,
                                                       float *__restrict__ out, int scaled) {
    __shared__ double r_o[FS_MAX_HANDS];
    __shared__ double u[52];
    __shared__ int cu[52];
    __shared__ double tot[kFsThreads / 32];
    __shared__ int ctot[kFsThreads / 32];
    const FsTermItem I = items[blockIdx.x];
    const int opp = 1 - trav;
    const int Ho = opp == 0 ? T.H0 : T.H1, Ht = trav == 0 ? T.H0 : T.H1;
    const size_t hs = static_cast<size_t>(T.HS);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    double f = 0.0;
    int cf = 0;
    for (int o = tid; o < Ho; o += blockDim.x) {
        const int code = T.hand_cards[opp * T.HS + o];
        const int x = code & 0xff, y = (code >> 8) & 0xff;
        bool blocked = false;
        for (int k = 0; k < I.nb; ++k) blocked |= x == I.board[k] || y == I.board[k];
        const double r = blocked ? 0.0 : static_cast<double>(reach[static_cast<size_t>(I.opp_row) * hs + o]);
        r_o[o] = blocked ? -1.0 : r;   // -1: the board blocks the hand
        f += r;
        cf += (!blocked && r > 0.0) ? 1 : 0;
    }
    for (int k = 16; k > 0; k >>= 1) {
        f += __shfl_xor_sync(0xffffffffu, f, k);
        cf += __shfl_xor_sync(0xffffffffu, cf, k);
    }
    if (lane == 0) {
        tot[warp] = f;
        ctot[warp] = cf;
    }
    __syncthreads();
    if (tid < 52) {
        double s = 0.0;
        int n = 0;
        const int *cl = T.f_clist + opp * 2 * T.HS;
        for (int k = T.f_coff[opp * 53 + tid]; k < T.f_coff[opp * 53 + tid + 1]; ++k) {
            const double r = r_o[cl[k]];
            if (r >= 0.0) {
                s += r;
                n += r > 0.0 ? 1 : 0;
            }
        }
        u[tid] = s;
        cu[tid] = n;
    }
    __syncthreads();
    double F = 0.0;
    int CF = 0;
    for (int w = 0; w < kFsThreads / 32; ++w) {
        F += tot[w];
        CF += ctot[w];
    }
    const float sc = scaled ? I.scale : 1.0f;
    const int *cl = T.f_clist + opp * 2 * T.HS;
    for (int h = tid; h < Ht; h += blockDim.x) {
        const int code = T.hand_cards[trav * T.HS + h];
        const int a = code & 0xff, b = (code >> 8) & 0xff;
        double same = 0.0;
        int csame = 0;
        for (int k = T.f_coff[opp * 53 + a]; k < T.f_coff[opp * 53 + a + 1]; ++k) {
            const int o = cl[k];
            const int oc = T.hand_cards[opp * T.HS + o];
            if ((oc & 0xff) != b && ((oc >> 8) & 0xff) != b) continue;
            const double r = r_o[o];
            if (r >= 0.0) {
                same += r;
                csame += r > 0.0 ? 1 : 0;
            }
        }
        const int cnt = CF - cu[a] - cu[b] + csame;
        const double mass = cnt == 0 ? 0.0 : F - u[a] - u[b] + same;
        out[static_cast<size_t>(I.node) * hs + h] = static_cast<float>(mass) * I.payoff * sc;
    }
}

// Showdowns (flop_solve.cu:781-833): +-half_pot per opponent hand that is
// weaker / stronger, ties 0, hands the board blocks 0.  With the opponent's
// hands in ascending strength on this river board, W = the reach below the
// traverser hand's strength and L = above it, each less the opponent hands
// holding one of its two cards (their own prefix sums along each card's
// list); value = (W - L) x half_pot, FP64 sums.  The same on 0/1 counts
// gives exactly 0 where no positive-reach opponent hand wins or loses.
__global__ void __launch_bounds__(kFsThreads) k_fs_showdown(const FsTermItem *__restrict__ items, int trav,
                                                           const float *__restrict__ reach, FsTables T,
                                                           float *__restrict__ out, int scaled) {
    __shared__ double P[FS_MAX_HANDS + 1];
    __shared__ int Pc[FS_MAX_HANDS + 1];
    __shared__ double PC[2 * FS_MAX_HANDS + 52];
    __shared__ int PCc[2 * FS_MAX_HANDS + 52];
    __shared__ double x_s[FS_MAX_HANDS];
    const FsTermItem I = items[blockIdx.x];
    const int opp = 1 - trav;
    const int Ho = opp == 0 ? T.H0 : T.H1, Ht = trav == 0 ? T.H0 : T.H1;
    const size_t hs = static_cast<size_t>(T.HS);
    const int tid = threadIdx.x, lane = tid & 31;
    const size_t bo = static_cast<size_t>(I.sboard) * 2 + opp, bt = static_cast<size_t>(I.sboard) * 2 + trav;
    const int *ord = T.sd_ord + bo * hs;
    const unsigned *so = T.sd_str + bo * hs;
    // the opponent's reach by position (0 where the board blocks the hand)
    for (int k = tid; k < Ho; k += blockDim.x) {
        const int o = ord[k];
        x_s[k] = so[o] == 0u ? 0.0 : static_cast<double>(reach[static_cast<size_t>(I.opp_row) * hs + o]);
    }
    __syncthreads();
    if (tid < 32) {
        // prefix sums over positions: each lane a run of consecutive
        // positions, lane totals scanned across the warp (fixed order)
        constexpr int kRun = (FS_MAX_HANDS + 31) / 32;
        const int k0 = lane * kRun;
        double s = 0.0;
        int n = 0;
        for (int i = 0; i < kRun; ++i)
            if (k0 + i < Ho) {
                s += x_s[k0 + i];
                n += x_s[k0 + i] > 0.0 ? 1 : 0;
            }
        double incl = s;
        int nincl = n;
        for (int d = 1; d < 32; d <<= 1) {
            const double v = __shfl_up_sync(0xffffffffu, incl, d);
            const int m = __shfl_up_sync(0xffffffffu, nincl, d);
            if (lane >= d) {
                incl += v;
                nincl += m;
            }
        }
        double run = incl - s;
        int nrun = nincl - n;
        for (int i = 0; i < kRun; ++i)
            if (k0 + i < Ho) {
                P[k0 + i] = run;
                Pc[k0 + i] = nrun;
                run += x_s[k0 + i];
                nrun += x_s[k0 + i] > 0.0 ? 1 : 0;
            }
        if (lane == 31) {
            P[Ho] = incl;
            Pc[Ho] = nincl;
        }
    } else if (tid >= 64 && tid < 64 + 52) {
        // per card: prefix sums along the opponent's hands holding it
        const int c = tid - 64;
        const int *coff = T.sd_coff + bo * 53;
        const int *cl = T.sd_clist + bo * 2 * hs;
        const int base = coff[c] + c;
        double s = 0.0;
        int n = 0;
        PC[base] = 0.0;
        PCc[base] = 0;
        for (int k = coff[c]; k < coff[c + 1]; ++k) {
            const double v = x_s[cl[k]];
            s += v;
            n += v > 0.0 ? 1 : 0;
            PC[base + (k - coff[c]) + 1] = s;
            PCc[base + (k - coff[c]) + 1] = n;
        }
    }
    __syncthreads();
    const float sc = scaled ? I.scale : 1.0f;
    const unsigned *st = T.sd_str + bt * hs;
    const int *coff = T.sd_coff + bo * 53;
    for (int h = tid; h < Ht; h += blockDim.x) {
        float v = 0.f;
        if (st[h] != 0u) {
            const int4 hp = reinterpret_cast<const int4 *>(T.sd_hpos)[bt * hs + h];
            const int lo = hp.x & 0xffff, hi = hp.x >> 16;
            const int c1 = hp.y & 0xff, c2 = (hp.y >> 8) & 0xff;
            const int b1 = coff[c1] + c1, n1 = coff[c1 + 1] - coff[c1];
            const int b2 = coff[c2] + c2, n2 = coff[c2 + 1] - coff[c2];
            const int l1lo = hp.z & 0xffff, l1hi = hp.z >> 16, l2lo = hp.w & 0xffff, l2hi = hp.w >> 16;
            const double W = P[lo] - PC[b1 + l1lo] - PC[b2 + l2lo];
            const double L = (P[Ho] - P[hi]) - (PC[b1 + n1] - PC[b1 + l1hi]) - (PC[b2 + n2] - PC[b2 + l2hi]);
            const int cw = Pc[lo] - PCc[b1 + l1lo] - PCc[b2 + l2lo];
            const int closs = (Pc[Ho] - Pc[hi]) - (PCc[b1 + n1] - PCc[b1 + l1hi]) - (PCc[b2 + n2] - PCc[b2 + l2hi]);
            const double w = cw == 0 ? 0.0 : W, l = closs == 0 ? 0.0 : L;
            v = static_cast<float>((w - l) * static_cast<double>(I.half_pot));
        }
        out[static_cast<size_t>(I.node) * hs + h] = v * sc;
    }
}

// the regret-matched strategy of every decision node of player p into
// sig [E][HS] (the read-out keeps the last pass's strategy)
__global__ void k_fs_sigma(const float *__restrict__ R, const int *__restrict__ edge_first,
                           const int *__restrict__ edge_na, int E, int HS, int H, float *__restrict__ sig) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= E * HS) return;
    const int e = i / HS, h = i - e * HS;
    if (h >= H) return;
    const int fe = edge_first[e], na = edge_na[e];
    float sum = 0.f;
    for (int a = 0; a < na; ++a) {
        const float r = R[static_cast<size_t>(fe + a) * HS + h];
        sum += r > 0.f ? r : 0.f;
    }
    const float r = R[i];
    sig[i] = sum > 0.f ? (r > 0.f ? r : 0.f) * (1.0f / sum) : 1.0f / static_cast<float>(na);
}

// one level of the read-out: every node's value for traverser t from its
// children (terminals were written by k_fs_fold / k_fs_showdown): the traverser's decisions
// weight by its last-pass strategy, the opponent's sum, chance nodes average
// (flop_solve.cu:835-892 order: children in order, then the division)
__global__ void k_fs_value_level(const FSNode *__restrict__ nodes, const int *__restrict__ children,
                                 const int *__restrict__ lev, int n, const int *__restrict__ first_edge,
                                 const float *__restrict__ sig, int trav, int HS, int H, float *__restrict__ val) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * HS) return;
    const int x = lev[i / HS], h = i % HS;
    if (h >= H) return;
    const FSNode nd = nodes[x];
    if (nd.type != FS_NODE_DECISION && nd.type != FS_NODE_CHANCE) return;
    const size_t hs = static_cast<size_t>(HS);
    float v = 0.f;
    for (int a = 0; a < nd.num_children; ++a) {
        const float cv = val[static_cast<size_t>(children[nd.first_child + a]) * hs + h];
        if (nd.type == FS_NODE_DECISION && nd.player == trav)
            v += sig[static_cast<size_t>(first_edge[x] + a) * hs + h] * cv;
        else
            v += cv;
    }
    if (nd.type == FS_NODE_CHANCE) v = v / static_cast<float>(nd.num_children);
    val[static_cast<size_t>(x) * hs + h] = v;
}

#define FCK(call)                                                                     \
    do {                                                                              \
        cudaError_t e_ = (call);                                                      \
        if (e_ != cudaSuccess) {                                                      \
            set_error(std::string("CUDA: ") + cudaGetErrorString(e_) + " at " #call); \
            return e_ == cudaErrorMemoryAllocation ? SS_ERR_NOMEM : SS_ERR_CUDA;      \
        }                                                                             \
    } while (0)

struct Blob {
    std::vector<char> host;
    size_t add(const void *src, size_t bytes) {
        size_t off = (host.size() + 255) & ~static_cast<size_t>(255);
        host.resize(off + bytes);
        if (bytes && src) std::memcpy(host.data() + off, src, bytes);
        return off;
    }
    template <class T>
    size_t add(const std::vector<T> &v) {
        return add(v.data(), v.size() * sizeof(T));
    }
};

// one solve's device state and launch lists
class Solve {
  public:
    FsPlan P;
    cudaStream_t stream = nullptr;
    char *dbase = nullptr;
    float *dstate = nullptr;
    int *diter = nullptr;
    float *dsnap = nullptr;
    float *dsig = nullptr, *dval = nullptr;   // read-out
    DevCtx c{};
    const ReachItem *reach_items[2] = {};
    std::vector<std::pair<int, int>> reach_lv[2], cfv_lv[2];
    const CfvItem *cfv_items[2] = {};
    const FsTermItem *term_items[2] = {};
    const int *hand_cards = nullptr, *edge_first = nullptr, *edge_na = nullptr, *depth_nodes = nullptr;
    FsTables tab{};
    FSNode *dnodes = nullptr;
    int *dchildren = nullptr;
    const int *dfirst_edge = nullptr;
    cudaGraphExec_t gblock = nullptr;
    int block_iters = 10;

    ~Solve() {
        if (gblock) cudaGraphExecDestroy(gblock);
        if (stream) {
            for (void *p : {static_cast<void *>(dbase), static_cast<void *>(dstate),
                            static_cast<void *>(diter), static_cast<void *>(dsnap), static_cast<void *>(dsig),
                            static_cast<void *>(dval), static_cast<void *>(dnodes), static_cast<void *>(dchildren)})
                if (p) cudaFreeAsync(p, stream);
            cudaStreamSynchronize(stream);
            cudaStreamDestroy(stream);
        }
    }

    int init(const FSTreeData &td) {
        int rc = build_plan(td, &P);
        if (rc != SS_OK) return rc;
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
            set_error("no CUDA device");
            return SS_ERR_NO_DEVICE;
        }
        FCK(cudaSetDevice(0));
        FCK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        const size_t HS = static_cast<size_t>(P.HS), E = static_cast<size_t>(P.E), N = static_cast<size_t>(P.N);
        Blob b;
        size_t o_reach[2], o_cfv[2], o_term[2];
        for (int p = 0; p < 2; ++p) {
            std::vector<ReachItem> all;
            for (auto &lv : P.reach_levels[p]) {
                reach_lv[p].push_back({static_cast<int>(all.size()), static_cast<int>(lv.size())});
                all.insert(all.end(), lv.begin(), lv.end());
            }
            o_reach[p] = b.add(all);
            std::vector<CfvItem> call;
            for (auto &lv : P.cfv_levels[p]) {
                cfv_lv[p].push_back({static_cast<int>(call.size()), static_cast<int>(lv.size())});
                call.insert(call.end(), lv.begin(), lv.end());
            }
            o_cfv[p] = b.add(call);
            o_term[p] = b.add(P.term[p]);
        }
        std::vector<int> ef(E), ena(E);
        for (size_t e = 0; e < E; ++e) {
            ef[e] = P.first_edge[P.edge_node[e]];
            ena[e] = td.nodes[P.edge_node[e]].num_children;
        }
        const size_t o_fro = b.add(P.fr_off), o_fri = b.add(P.fr_items), o_hc = b.add(P.hand_cards),
                     o_ef = b.add(ef), o_ena = b.add(ena), o_dn = b.add(P.depth_nodes), o_fe = b.add(P.first_edge),
                     o_fco = b.add(P.f_coff), o_fcl = b.add(P.f_clist), o_sst = b.add(P.sd_str),
                     o_sor = b.add(P.sd_ord), o_shp = b.add(P.sd_hpos), o_sco = b.add(P.sd_coff),
                     o_scl = b.add(P.sd_clist);
        FCK(cudaMallocAsync(reinterpret_cast<void **>(&dbase), std::max<size_t>(b.host.size(), 256), stream));
        FCK(cudaMemcpyAsync(dbase, b.host.data(), b.host.size(), cudaMemcpyHostToDevice, stream));
        for (int p = 0; p < 2; ++p) {
            reach_items[p] = reinterpret_cast<const ReachItem *>(dbase + o_reach[p]);
            cfv_items[p] = reinterpret_cast<const CfvItem *>(dbase + o_cfv[p]);
            term_items[p] = reinterpret_cast<const FsTermItem *>(dbase + o_term[p]);
        }
        hand_cards = reinterpret_cast<const int *>(dbase + o_hc);
        tab.hand_cards = hand_cards;
        tab.f_coff = reinterpret_cast<const int *>(dbase + o_fco);
        tab.f_clist = reinterpret_cast<const int *>(dbase + o_fcl);
        tab.sd_str = reinterpret_cast<const unsigned *>(dbase + o_sst);
        tab.sd_ord = reinterpret_cast<const int *>(dbase + o_sor);
        tab.sd_hpos = reinterpret_cast<const int *>(dbase + o_shp);
        tab.sd_coff = reinterpret_cast<const int *>(dbase + o_sco);
        tab.sd_clist = reinterpret_cast<const int *>(dbase + o_scl);
        tab.HS = P.HS;
        tab.H0 = P.H[0];
        tab.H1 = P.H[1];
        edge_first = reinterpret_cast<const int *>(dbase + o_ef);
        edge_na = reinterpret_cast<const int *>(dbase + o_ena);
        depth_nodes = reinterpret_cast<const int *>(dbase + o_dn);
        dfirst_edge = reinterpret_cast<const int *>(dbase + o_fe);
        // state: regrets, strategy sums, reach (weights in the last 2 rows), values
        const size_t nR = E * HS, nReach = (E + 2) * HS, nVal = N * HS;
        FCK(cudaMallocAsync(reinterpret_cast<void **>(&dstate), (2 * nR + nReach + nVal) * sizeof(float), stream));
        FCK(cudaMemsetAsync(dstate, 0, (2 * nR + nReach + nVal) * sizeof(float), stream));
        c.R = dstate;
        c.S = c.R + nR;
        c.reach = c.S + nR;
        c.val = c.reach + nReach;
        std::vector<float> w(2 * HS, 0.f);
        for (int p = 0; p < 2; ++p)
            for (int h = 0; h < P.H[p]; ++h) w[p * HS + h] = td.weights[p][h];
        FCK(cudaMemcpyAsync(c.reach + E * HS, w.data(), w.size() * sizeof(float), cudaMemcpyHostToDevice, stream));
        FCK(cudaMallocAsync(reinterpret_cast<void **>(&diter), sizeof(int), stream));
        FCK(cudaMemsetAsync(diter, 0, sizeof(int), stream));
        const int nrs = P.root_na * std::max(1, P.H[P.root_player]);
        FCK(cudaMallocAsync(reinterpret_cast<void **>(&dsnap), nrs * sizeof(float), stream));
        FCK(cudaMemsetAsync(dsnap, 0, nrs * sizeof(float), stream));
        c.fr_off = reinterpret_cast<const int *>(dbase + o_fro);
        c.fr_items = reinterpret_cast<const int *>(dbase + o_fri);
        c.iter = diter;
        c.HS = P.HS;
        c.np = 2;
        c.H[0] = P.H[0];
        c.H[1] = P.H[1];
        FCK(cudaStreamSynchronize(stream));   // host staging must outlive the copies
        // all regrets 0: uniform play
        for (int p = 0; p < 2; ++p) FCK(reach(p));
        return SS_OK;
    }

    cudaError_t reach(int p) {
        for (auto &lv : reach_lv[p]) {
            cudaError_t e = launch_reach(c, reach_items[p] + lv.first, lv.second, P.H[p], stream);
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    }

    cudaError_t terms(int t, float *out, int scaled) {
        const int nf = P.nfold[t], ns = static_cast<int>(P.term[t].size()) - nf;
        if (nf > 0) k_fs_fold<<<nf, kFsThreads, 0, stream>>>(term_items[t], t, c.reach, tab, out, scaled);
        if (ns > 0) k_fs_showdown<<<ns, kFsThreads, 0, stream>>>(term_items[t] + nf, t, c.reach, tab, out, scaled);
        return cudaGetLastError();
    }

    // one iteration: per traverser terminals, values and regrets bottom-up,
    // then its reach; the root strategy is taken before the last traverser's
    // pass (the reference's last regret matching)
    cudaError_t iteration(bool keep_sigma) {
        cudaError_t e = launch_bump(diter, stream);
        for (int t = 0; t < 2 && e == cudaSuccess; ++t) {
            if (t == 1) {
                e = launch_root_strategy(c, P.first_edge[0], P.root_na, -1, P.H[P.root_player], dsnap, stream);
                if (e == cudaSuccess && keep_sigma && P.E > 0) {
                    const int n = P.E * P.HS;
                    k_fs_sigma<<<(n + 255) / 256, 256, 0, stream>>>(c.R, edge_first, edge_na, P.E, P.HS, P.H[1], dsig);
                    e = cudaGetLastError();
                }
            }
            if (e == cudaSuccess) e = terms(t, c.val, 1);
            for (size_t l = 0; l < cfv_lv[t].size() && e == cudaSuccess; ++l)
                e = launch_cfv(c, cfv_items[t] + cfv_lv[t][l].first, cfv_lv[t][l].second, P.cfv_nlong[t][l], P.H[t],
                               stream);
            if (e == cudaSuccess) e = reach(t);
        }
        return e;
    }

    int run(int iters, bool keep_sigma_last) {
        int done = 0;
        const int graph_part = keep_sigma_last ? iters - 1 : iters;
        if (graph_part >= block_iters) {
            cudaGraph_t g = nullptr;
            FCK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
            cudaError_t body = cudaSuccess;
            for (int i = 0; i < block_iters && body == cudaSuccess; ++i) body = iteration(false);
            cudaError_t e = cudaStreamEndCapture(stream, &g);
            if (body != cudaSuccess) {
                if (g) cudaGraphDestroy(g);
                FCK(body);
            }
            FCK(e);
            e = cudaGraphInstantiate(&gblock, g, 0);
            cudaGraphDestroy(g);
            FCK(e);
            for (; done + block_iters <= graph_part; done += block_iters) FCK(cudaGraphLaunch(gblock, stream));
        }
        for (; done < iters; ++done) FCK(iteration(keep_sigma_last && done == iters - 1));
        FCK(cudaStreamSynchronize(stream));
        return SS_OK;
    }

    // the last traverser's value at every node under the last pass's strategy
    int readout() {
        const int t = 1;
        FCK(terms(t, dval, 0));
        const int L = static_cast<int>(P.depth_off.size()) - 1;
        for (int l = 0; l < L; ++l) {
            const int n = P.depth_off[l + 1] - P.depth_off[l];
            const int tot = n * P.HS;
            k_fs_value_level<<<(tot + 255) / 256, 256, 0, stream>>>(dnodes, dchildren, depth_nodes + P.depth_off[l], n,
                                                                   dfirst_edge, dsig, t, P.HS, P.H[t], dval);
            FCK(cudaGetLastError());
        }
        FCK(cudaStreamSynchronize(stream));
        return SS_OK;
    }
};

}  // namespace

int solve(FSTreeData *td, int iterations, FSOutput *out, bool extract) {
    std::memset(out, 0, sizeof(*out));
    if (!td) {
        set_error("fs_solve_gpu: no tree");
        return SS_ERR_INVALID;
    }
    if (iterations < 1) {
        set_error("fs_solve_gpu: max_iterations must be >= 1");
        return SS_ERR_INVALID;
    }
    Solve s;
    int rc = s.init(*td);
    if (rc != SS_OK) return rc;
    const FsPlan &P = s.P;
    const size_t HS = static_cast<size_t>(P.HS), N = static_cast<size_t>(P.N), mh = static_cast<size_t>(P.max_h);
    if (extract) {
        FCK(cudaMallocAsync(reinterpret_cast<void **>(&s.dsig), std::max<size_t>(1, P.E * HS) * sizeof(float), s.stream));
        FCK(cudaMemsetAsync(s.dsig, 0, std::max<size_t>(1, P.E * HS) * sizeof(float), s.stream));
        FCK(cudaMallocAsync(reinterpret_cast<void **>(&s.dval), N * HS * sizeof(float), s.stream));
        FCK(cudaMemsetAsync(s.dval, 0, N * HS * sizeof(float), s.stream));
        FCK(cudaMallocAsync(reinterpret_cast<void **>(&s.dnodes), N * sizeof(FSNode), s.stream));
        FCK(cudaMemcpyAsync(s.dnodes, td->nodes, N * sizeof(FSNode), cudaMemcpyHostToDevice, s.stream));
        FCK(cudaMallocAsync(reinterpret_cast<void **>(&s.dchildren),
                            std::max(1, td->num_children_total) * sizeof(int), s.stream));
        FCK(cudaMemcpyAsync(s.dchildren, td->children, td->num_children_total * sizeof(int), cudaMemcpyHostToDevice,
                            s.stream));
    }
    rc = s.run(iterations, extract);
    if (rc != SS_OK) return rc;
    const int nrh = P.H[P.root_player];
    FSOutput o{};
    o.root_num_actions = P.root_na;
    o.root_player = P.root_player;
    o.root_strategy = static_cast<float *>(std::malloc(std::max(1, P.root_na * nrh) * sizeof(float)));
    if (!o.root_strategy) {
        set_error("fs_solve_gpu: out of host memory");
        return SS_ERR_NOMEM;
    }
    FCK(cudaMemcpy(o.root_strategy, s.dsnap, P.root_na * nrh * sizeof(float), cudaMemcpyDeviceToHost));
    if (extract) {
        rc = s.readout();
        if (rc != SS_OK) {
            free_output(&o);
            return rc;
        }
        o.max_hands = P.max_h;
        o.all_avg_strategies = static_cast<float *>(std::calloc(N * FS_MAX_ACTIONS * mh, sizeof(float)));
        o.all_cfv = static_cast<float *>(std::malloc(std::max<size_t>(1, N * mh) * sizeof(float)));
        std::vector<float> S(P.E * HS), V(N * HS);
        if (!o.all_avg_strategies || !o.all_cfv) {
            free_output(&o);
            set_error("fs_solve_gpu_extract_all: out of host memory");
            return SS_ERR_NOMEM;
        }
        FCK(cudaMemcpy(S.data(), s.c.S, S.size() * sizeof(float), cudaMemcpyDeviceToHost));
        FCK(cudaMemcpy(V.data(), s.dval, V.size() * sizeof(float), cudaMemcpyDeviceToHost));
        for (size_t x = 0; x < N; ++x)
            for (size_t h = 0; h < mh; ++h) o.all_cfv[x * mh + h] = h < static_cast<size_t>(P.H[1]) ? V[x * HS + h] : 0.f;
        // normalised strategy sums at every decision node (flop_solve.cu:1516-1540)
        for (int x : P.dec_nodes) {
            const FSNode &n = td->nodes[x];
            const int fe = P.first_edge[x], na = n.num_children;
            float *dst = o.all_avg_strategies + static_cast<size_t>(x) * FS_MAX_ACTIONS * mh;
            for (int h = 0; h < P.H[n.player]; ++h) {
                float sum = 0.f;
                for (int a = 0; a < na; ++a) {
                    const float v = S[(fe + a) * HS + h];
                    sum += v > 0.f ? v : 0.f;
                }
                for (int a = 0; a < na; ++a) {
                    const float v = S[(fe + a) * HS + h];
                    dst[a * mh + h] = sum > 0.f ? (v > 0.f ? v * (1.0f / sum) : 0.f) : 1.0f / static_cast<float>(na);
                }
            }
        }
        // turn roots: the decision children of the flop-ending chance nodes
        std::vector<int> roots, cards;
        for (int x = 0; x < P.N; ++x) {
            const FSNode &n = td->nodes[x];
            if (n.type != FS_NODE_CHANCE || n.num_board != 3) continue;
            for (int a = 0; a < n.num_children; ++a) {
                const int ch = td->children[n.first_child + a];
                if (td->nodes[ch].type == FS_NODE_DECISION) {
                    roots.push_back(ch);
                    cards.push_back(td->nodes[ch].board_cards[3]);
                }
            }
        }
        o.turn_root_indices = static_cast<int *>(std::malloc(std::max<size_t>(1, roots.size()) * sizeof(int)));
        o.turn_root_cards = static_cast<int *>(std::malloc(std::max<size_t>(1, roots.size()) * sizeof(int)));
        if (!o.turn_root_indices || !o.turn_root_cards) {
            free_output(&o);
            set_error("fs_solve_gpu_extract_all: out of host memory");
            return SS_ERR_NOMEM;
        }
        std::copy(roots.begin(), roots.end(), o.turn_root_indices);
        std::copy(cards.begin(), cards.end(), o.turn_root_cards);
        o.num_turn_roots = static_cast<int>(roots.size());
    }
    *out = o;
    return SS_OK;
}

void free_output(FSOutput *o) {
    if (!o) return;
    std::free(o->root_strategy);
    std::free(o->root_ev);
    std::free(o->all_avg_strategies);
    std::free(o->all_cfv);
    std::free(o->turn_root_indices);
    std::free(o->turn_root_cards);
    std::memset(o, 0, sizeof(*o));
}

}  // namespace fs
}  // namespace ssb
