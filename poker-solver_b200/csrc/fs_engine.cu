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
            P.cfv_levels[t][h].push_back(it);
        }
        P.cfv_nlong[t].assign(P.cfv_levels[t].size(), 0);
        for (size_t l = 0; l < P.cfv_levels[t].size(); ++l) {
            auto &v = P.cfv_levels[t][l];
            auto is_short = [&](const CfvItem &it) {
                return P.fr_off[it.first_edge + it.na] - P.fr_off[it.first_edge] < kCfvLongFrontier;
            };
            auto mid = std::stable_partition(v.begin(), v.end(), is_short);
            P.cfv_nlong[t][l] = static_cast<int>(v.end() - mid);
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
    }
    // hands
    P.hand_cards.assign(2 * static_cast<size_t>(P.HS), -1);
    for (int p = 0; p < 2; ++p)
        for (int h = 0; h < P.H[p]; ++h) P.hand_cards[p * P.HS + h] = td.hands[p][h][0] | (td.hands[p][h][1] << 8);
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

// strengths [nsb][2][HS] of both players' hands on every showdown board
// (0: the board blocks the hand)
__global__ void k_fs_strengths(const int *__restrict__ sboards, int nsb, const int *__restrict__ hand_cards, int HS,
                               int H0, int H1, unsigned *__restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nsb * 2 * HS) return;
    const int b = i / (2 * HS), r = i - b * 2 * HS, p = r / HS, h = r - p * HS;
    unsigned s = 0;
    if (h < (p == 0 ? H0 : H1)) {
        const int code = hand_cards[p * HS + h];
        int c[7] = {sboards[5 * b], sboards[5 * b + 1], sboards[5 * b + 2], sboards[5 * b + 3], sboards[5 * b + 4],
                    code & 0xff, (code >> 8) & 0xff};
        bool clash = false;
        for (int k = 0; k < 5; ++k) clash |= c[k] == c[5] || c[k] == c[6];
        s = clash ? 0u : rank7(c);
    }
    out[i] = s;
}

// one block per terminal (flop_solve.cu:731-833 semantics): the opponent's
// reach row, cards and strengths staged in shared memory, one traverser hand
// per thread, opponent hands summed in hand order
__global__ void __launch_bounds__(kFsThreads) k_fs_term(const FsTermItem *__restrict__ items, int trav,
                                                       const float *__restrict__ reach,
                                                       const int *__restrict__ hand_cards,
                                                       const unsigned *__restrict__ str, int HS, int H0, int H1,
                                                       float *__restrict__ out, int scaled) {
    __shared__ float r_o[FS_MAX_HANDS];
    __shared__ int c_o[FS_MAX_HANDS];
    __shared__ unsigned s_o[FS_MAX_HANDS];
    const FsTermItem I = items[blockIdx.x];
    const int opp = 1 - trav;
    const int Ho = opp == 0 ? H0 : H1, Ht = trav == 0 ? H0 : H1;
    const size_t hs = static_cast<size_t>(HS);
    for (int o = threadIdx.x; o < Ho; o += blockDim.x) {
        const int code = hand_cards[opp * HS + o];
        const int a = code & 0xff, b = (code >> 8) & 0xff;
        r_o[o] = reach[static_cast<size_t>(I.opp_row) * hs + o];
        bool blocked = false;
        if (I.kind == 0)
            for (int k = 0; k < I.nb; ++k) blocked |= a == I.board[k] || b == I.board[k];
        c_o[o] = blocked ? -1 : code;   // a fold skips opponent hands the node's board blocks
        s_o[o] = I.kind == 1 ? str[(static_cast<size_t>(I.sboard) * 2 + opp) * hs + o] : 0u;
    }
    __syncthreads();
    const float sc = scaled ? I.scale : 1.0f;
    for (int h = threadIdx.x; h < Ht; h += blockDim.x) {
        const int code = hand_cards[trav * HS + h];
        const int a = code & 0xff, b = (code >> 8) & 0xff;
        float v = 0.f;
        if (I.kind == 0) {
            float s = 0.f;
            for (int o = 0; o < Ho; ++o) {
                const int oc = c_o[o];
                if (oc < 0) continue;
                const int x = oc & 0xff, y = (oc >> 8) & 0xff;
                if (a == x || a == y || b == x || b == y) continue;
                s += r_o[o];
            }
            v = s * I.payoff;
        } else {
            const unsigned hsv = str[(static_cast<size_t>(I.sboard) * 2 + trav) * hs + h];
            if (hsv != 0u) {
                for (int o = 0; o < Ho; ++o) {
                    const int oc = c_o[o];
                    const int x = oc & 0xff, y = (oc >> 8) & 0xff;
                    if (a == x || a == y || b == x || b == y) continue;
                    const unsigned os = s_o[o];
                    if (os == 0u) continue;
                    const float wgt = r_o[o];
                    if (hsv > os)
                        v += wgt * I.half_pot;
                    else if (hsv < os)
                        v -= wgt * I.half_pot;
                }
            }
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
// children (terminals were written by k_fs_term): the traverser's decisions
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
    unsigned *dstr = nullptr;
    int *diter = nullptr;
    float *dsnap = nullptr;
    float *dsig = nullptr, *dval = nullptr;   // read-out
    DevCtx c{};
    const ReachItem *reach_items[2] = {};
    std::vector<std::pair<int, int>> reach_lv[2], cfv_lv[2];
    const CfvItem *cfv_items[2] = {};
    const FsTermItem *term_items[2] = {};
    const int *hand_cards = nullptr, *edge_first = nullptr, *edge_na = nullptr, *depth_nodes = nullptr;
    FSNode *dnodes = nullptr;
    int *dchildren = nullptr;
    const int *dfirst_edge = nullptr;
    cudaGraphExec_t gblock = nullptr;
    int block_iters = 10;

    ~Solve() {
        if (gblock) cudaGraphExecDestroy(gblock);
        if (stream) {
            for (void *p : {static_cast<void *>(dbase), static_cast<void *>(dstate), static_cast<void *>(dstr),
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
                     o_sb = b.add(P.sboards), o_ef = b.add(ef), o_ena = b.add(ena), o_dn = b.add(P.depth_nodes),
                     o_fe = b.add(P.first_edge);
        FCK(cudaMallocAsync(reinterpret_cast<void **>(&dbase), std::max<size_t>(b.host.size(), 256), stream));
        FCK(cudaMemcpyAsync(dbase, b.host.data(), b.host.size(), cudaMemcpyHostToDevice, stream));
        for (int p = 0; p < 2; ++p) {
            reach_items[p] = reinterpret_cast<const ReachItem *>(dbase + o_reach[p]);
            cfv_items[p] = reinterpret_cast<const CfvItem *>(dbase + o_cfv[p]);
            term_items[p] = reinterpret_cast<const FsTermItem *>(dbase + o_term[p]);
        }
        hand_cards = reinterpret_cast<const int *>(dbase + o_hc);
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
        const int nsb = static_cast<int>(P.sboards.size() / 5);
        FCK(cudaMallocAsync(reinterpret_cast<void **>(&dstr), std::max<size_t>(1, nsb * 2 * HS) * sizeof(unsigned),
                            stream));
        if (nsb > 0) {
            const int n = nsb * 2 * P.HS;
            k_fs_strengths<<<(n + 255) / 256, 256, 0, stream>>>(reinterpret_cast<const int *>(dbase + o_sb), nsb,
                                                                 hand_cards, P.HS, P.H[0], P.H[1], dstr);
            FCK(cudaGetLastError());
        }
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
        const int n = static_cast<int>(P.term[t].size());
        if (n == 0) return cudaSuccess;
        k_fs_term<<<n, kFsThreads, 0, stream>>>(term_items[t], t, c.reach, hand_cards, dstr, P.HS, P.H[0], P.H[1],
                                                out, scaled);
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
