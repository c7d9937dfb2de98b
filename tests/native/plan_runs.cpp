// Prints the three-way showdown sweep tables of build_plan as JSON, for
// tests/test_plan_runs.py: a 3-player river tree (bets {0.5, 1.0} + all-in,
// 2 raises) on the given board, each player's range a seeded random subset
// of the non-board combos (all of them when hands >= 1081).
//   plan_runs <seed> <hands> <board card x5>
#include "ss_engine.h"
#include "street_solve.h"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <string>
#include <vector>

namespace ssb {
// the engine's error channel lives in a CUDA translation unit; the planner
// alone needs these two
static std::string g_err;
void set_error(const std::string &s) { g_err = s; }
const char *last_error() { return g_err.c_str(); }
}  // namespace ssb

int main(int argc, char **argv) {
    if (argc != 8) return 2;
    const int seed = std::atoi(argv[1]), nh = std::atoi(argv[2]);
    int board[5];
    for (int i = 0; i < 5; ++i) board[i] = std::atoi(argv[3 + i]);
    float bets[2] = {0.5f, 1.0f};
    int order[3] = {0, 1, 2};
    ssb::BuiltTree bt;
    if (ssb::build_street_tree(board, 5, 300, 1000, bets, 2, 3, order, 1, 0, 2, &bt) != SS_OK) return 3;
    std::vector<int> all;
    for (int a = 0; a < 52; ++a)
        for (int b = a + 1; b < 52; ++b) {
            bool on = false;
            for (int i = 0; i < 5; ++i) on = on || board[i] == a || board[i] == b;
            if (!on) all.push_back(a * 52 + b);
        }
    std::mt19937 rng(seed);
    std::vector<int> hands[3];
    std::vector<float> w[3];
    for (int p = 0; p < 3; ++p) {
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
    pb.num_players = 3;
    for (int p = 0; p < 3; ++p) {
        pb.hands[p] = hands[p].data();
        pb.weights[p] = w[p].data();
        pb.num_hands[p] = static_cast<int>(w[p].size());
    }
    for (int i = 0; i < 5; ++i) pb.board[i] = board[i];
    pb.num_board = 5;
    pb.is_river = 1;
    pb.starting_pot = 300;
    ssb::Plan P;
    if (ssb::build_plan(pb, &P) != SS_OK) {
        std::fprintf(stderr, "%s\n", ssb::last_error());
        return 4;
    }
    std::printf("{\"ncomb\": %d, \"chunks\": %d, \"slots\": %d, \"seg_cost\": %d, \"run_cost\": %d, \"spans\": [", P.ncomb,
                ssb::kSd2Chunks, ssb::kSd2Slots, ssb::kSd2SegCost, ssb::kSd2RunCost);
    for (int lg = 0; lg < ssb::kSd2Merge; ++lg) std::printf("%s%d", lg ? ", " : "", P.sd_span[lg]);
    std::printf("], \"players\": [");
    for (int p = 0; p < 3; ++p) {
        const int a = P.sd_seg_off[p], b = P.sd_seg_off[p + 1];
        // a segment holding one of the player's hands must be exactly one tie
        // group; the flag must match the hand table
        bool ok = true;
        for (int i = a; i < b; ++i) {
            const int lo = P.sd_seg[4 * i], hi = P.sd_seg[4 * i + 1], has = P.sd_seg[4 * i + 2];
            bool any = false;
            for (int q = lo; q < hi; ++q) any = any || P.pos_hand[static_cast<size_t>(p) * P.ncomb + q] >= 0;
            if (any != (has != 0)) ok = false;
            if (has && (P.sd_combo[lo].lo != lo || P.sd_combo[lo].hi != hi)) ok = false;
        }
        std::printf("%s{\"sd2_terminals\": %zu, \"flags_ok\": %s, \"segs\": [", p ? ", " : "", P.term[p][ssb::TK_SD2].size(),
                    ok ? "true" : "false");
        for (int i = a; i < b; ++i)
            std::printf("%s[%d, %d, %d]", i > a ? ", " : "", P.sd_seg[4 * i], P.sd_seg[4 * i + 1], P.sd_seg[4 * i + 2]);
        std::printf("], \"seg_base\": %d, \"chunk\": [", a);
        const int *ch = P.sd_chunk.data() + static_cast<size_t>(p) * (ssb::kSd2Chunks + 1);
        for (int k = 0; k <= ssb::kSd2Chunks; ++k) std::printf("%s%d", k ? ", " : "", ch[k]);
        std::printf("]}");
    }
    std::printf("]}\n");
    return 0;
}
