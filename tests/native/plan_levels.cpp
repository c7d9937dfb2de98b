// Checks the one-launch form of the value/regret levels that build_plan
// writes (short items, sliced items, slices, blocks) on a turn tree with
// continuation leaves, and prints the result as JSON for
// tests/test_plan_runs.py:
//   plan_levels <players> <hands> <raises> <board card x4>
#include "ss_engine.h"
#include "street_solve.h"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <random>
#include <string>
#include <vector>

namespace ssb {
static std::string g_err;
void set_error(const std::string &s) { g_err = s; }
const char *last_error() { return g_err.c_str(); }
}  // namespace ssb

static int fail(const std::string &why) {
    std::printf("{\"ok\": false, \"why\": \"%s\"}\n", why.c_str());
    return 0;
}

int main(int argc, char **argv) {
    if (argc != 8) return 2;
    const int np = std::atoi(argv[1]), nh = std::atoi(argv[2]), raises = std::atoi(argv[3]);
    int board[4];
    for (int i = 0; i < 4; ++i) board[i] = std::atoi(argv[4 + i]);
    float bets[3] = {0.33f, 0.75f, 1.5f};
    int order[6] = {0, 1, 2, 3, 4, 5};
    ssb::BuiltTree bt;
    if (ssb::build_street_tree(board, 4, 150, 500, bets, 3, np, order, 0, 1, raises, &bt) != SS_OK) return 3;
    std::vector<int> all;
    for (int a = 0; a < 52; ++a)
        for (int b = a + 1; b < 52; ++b) {
            bool on = false;
            for (int i = 0; i < 4; ++i) on = on || board[i] == a || board[i] == b;
            if (!on) all.push_back(a * 52 + b);
        }
    std::mt19937 rng(7);
    std::vector<int> hands[6];
    std::vector<float> w[6];
    for (int p = 0; p < np; ++p) {
        std::vector<int> pick = all;
        std::shuffle(pick.begin(), pick.end(), rng);
        pick.resize(std::min<size_t>(pick.size(), static_cast<size_t>(nh)));
        for (int c : pick) {
            hands[p].push_back(c / 52);
            hands[p].push_back(c % 52);
            w[p].push_back(std::uniform_real_distribution<float>(0.f, 1.f)(rng));
        }
    }
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
    for (int i = 0; i < 4; ++i) pb.board[i] = board[i];
    pb.num_board = 4;
    pb.is_river = 0;
    pb.starting_pot = 150;
    ssb::Plan P;
    if (ssb::build_plan(pb, &P) != SS_OK) {
        std::fprintf(stderr, "%s\n", ssb::last_error());
        return 4;
    }
    long long n_short = 0, n_long = 0, n_slices = 0, n_blocks = 0;
    std::vector<char> part_used(static_cast<size_t>(P.cfv_part_rows), 0), cnt_used(static_cast<size_t>(P.cfv_counters), 0);
    for (int t = 0; t < np; ++t) {
        const int nchunk = (P.H[t] + 63) / 64;
        const size_t nl = P.cfv_levels[t].size();
        if (P.cfv_short[t].size() != nl || P.cfv_long[t].size() != nl || P.cfv_slices[t].size() != nl ||
            P.cfv_blocks[t].size() != nl)
            return fail("level counts differ");
        for (size_t l = 0; l < nl; ++l) {
            // every item once, short or sliced by its frontier length
            std::map<int, int> seen;
            for (const auto &it : P.cfv_levels[t][l]) seen[it.node] += 1;
            for (const auto &it : P.cfv_short[t][l]) {
                if (P.fr_off[it.first_edge + it.na] - P.fr_off[it.first_edge] > ssb::kCfvShortRows)
                    return fail("long frontier in a short item");
                seen[it.node] -= 1;
            }
            for (const auto &L : P.cfv_long[t][l]) {
                const auto &it = L.it;
                if (P.fr_off[it.first_edge + it.na] - P.fr_off[it.first_edge] <= ssb::kCfvShortRows)
                    return fail("short frontier sliced");
                seen[it.node] -= 1;
                if (L.slot_off[0] != 0 || L.slot_off[it.na] != L.n_slices) return fail("slot offsets");
                for (int s = 0; s < L.n_slices; ++s) {
                    if (L.part_base + s >= P.cfv_part_rows || part_used[L.part_base + s]++) return fail("partial rows");
                }
                for (int ch = 0; ch < nchunk; ++ch)
                    if (L.cnt_base + ch >= P.cfv_counters || cnt_used[L.cnt_base + ch]++) return fail("counters");
            }
            for (auto &kv : seen)
                if (kv.second != 0) return fail("item coverage");
            // slices tile each edge's frontier in order, at most kCfvSliceRows rows each
            std::vector<std::vector<int>> next(P.cfv_long[t][l].size());
            std::vector<int> slot_next(P.cfv_long[t][l].size(), 0);
            for (size_t i = 0; i < P.cfv_long[t][l].size(); ++i) {
                const auto &L = P.cfv_long[t][l][i];
                next[i].assign(L.it.na, 0);
                for (int a = 0; a < L.it.na; ++a) next[i][a] = P.fr_off[L.it.first_edge + a];
            }
            for (const auto &S : P.cfv_slices[t][l]) {
                if (S.item < 0 || S.item >= static_cast<int>(P.cfv_long[t][l].size())) return fail("slice item");
                const auto &L = P.cfv_long[t][l][S.item];
                int a = 0;
                while (a < L.it.na && !(S.slot >= L.slot_off[a] && S.slot < L.slot_off[a + 1])) ++a;
                if (a == L.it.na) return fail("slice slot");
                if (S.slot != slot_next[S.item]++) return fail("slot order");
                if (S.k0 != next[S.item][a] || S.k1 <= S.k0 || S.k1 - S.k0 > ssb::kCfvSliceRows ||
                    S.k1 > P.fr_off[L.it.first_edge + a + 1])
                    return fail("slice rows");
                next[S.item][a] = S.k1;
            }
            for (size_t i = 0; i < P.cfv_long[t][l].size(); ++i) {
                const auto &L = P.cfv_long[t][l][i];
                if (slot_next[i] != L.n_slices) return fail("slice count");
                for (int a = 0; a < L.it.na; ++a)
                    if (next[i][a] != P.fr_off[L.it.first_edge + a + 1]) return fail("edge rows not covered");
            }
            // blocks: each short item and slice once per group of four chunks
            std::map<std::pair<int, int>, int> cover;
            for (const auto &B : P.cfv_blocks[t][l]) {
                if (B.chunk % 4 || B.chunk >= nchunk) return fail("block chunk");
                const int lim = B.kind == 0 ? static_cast<int>(P.cfv_short[t][l].size())
                                            : static_cast<int>(P.cfv_slices[t][l].size());
                if (B.index < 0 || B.index >= lim) return fail("block index");
                cover[{B.kind * 1000000 + B.index, B.chunk}] += 1;
            }
            const size_t want = (P.cfv_short[t][l].size() + P.cfv_slices[t][l].size()) * ((nchunk + 3) / 4);
            if (cover.size() != want) return fail("block coverage");
            for (auto &kv : cover)
                if (kv.second != 1) return fail("block repeated");
            n_short += static_cast<long long>(P.cfv_short[t][l].size());
            n_long += static_cast<long long>(P.cfv_long[t][l].size());
            n_slices += static_cast<long long>(P.cfv_slices[t][l].size());
            n_blocks += static_cast<long long>(P.cfv_blocks[t][l].size());
        }
    }
    for (char u : part_used)
        if (!u) return fail("unused partial row");
    for (char u : cnt_used)
        if (!u) return fail("unused counter");
    std::printf("{\"ok\": true, \"short\": %lld, \"long\": %lld, \"slices\": %lld, \"blocks\": %lld}\n", n_short, n_long,
                n_slices, n_blocks);
    return 0;
}
