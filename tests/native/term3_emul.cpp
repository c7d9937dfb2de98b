// Runs the three-opponent terminal blocks (k_term_cr3, k_term_sd3) on the
// host -- their phases over 256 emulated threads and the same per-thread
// steps (poker-solver_b200/csrc/ss_cr3.cuh) in the kernels' order -- over the
// work items the planner (ss_plan.cpp) makes for a seeded 4-player subgame,
// and compares every traverser hand with brute-force enumeration of the
// opponents' disjoint hand tuples, for tests/test_cr3_host.py.  This checks
// the kernels' use of the plan's tables (hand codes, pair tables, rank
// positions, tie groups, term groups) without a GPU.
//   term3_emul <seed> <board cards: 4 turn, 5 river> <hands per player> <zero fraction> <max items per traverser>
// Reach rows get random weights (some zero); turn leaves get random values.
// Prints JSON: items and hands checked, the largest relative error, and the
// hands whose enumerated value is exactly 0 but whose computed one is not.
#include "ss_cr3.cuh"
#include "ss_engine.h"
#include "street_solve.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <string>
#include <vector>

namespace ssb {
static std::string g_err;
void set_error(const std::string &s) { g_err = s; }
const char *last_error() { return g_err.c_str(); }
}  // namespace ssb

using namespace ssb;
using namespace ssb::cr3;

namespace {

struct Block {
    std::vector<double> A, B, P, PT, uA, uB, w, d, sc, r3;
    std::vector<int> iuA, iuB, iw, id, p3;
    std::vector<unsigned long long> mA, mB;
    std::vector<long long> isc;
    std::vector<unsigned short> xy;
    Tables t;
    explicit Block(int HS)
        : A(kS * kS), B(kS * kS), P(kS * kS), PT(kS * kS), uA(kS), uB(kS), w(kS), d(kS), sc(8), r3(HS),
          iuA(kS), iuB(kS), iw(kS), id(kS), p3(HS), mA(kS), mB(kS), isc(8), xy(HS) {
        t = Tables{A.data(), B.data(), P.data(), PT.data(), uA.data(), uB.data(), w.data(), d.data(),
                   iuA.data(), iuB.data(), iw.data(), id.data(), mA.data(), mB.data(), r3.data(), xy.data(),
                   sc.data(), isc.data()};
    }
};

constexpr int kNt = 256;

}  // namespace

int main(int argc, char **argv) {
    if (argc != 6) return 2;
    const unsigned seed = static_cast<unsigned>(std::atoi(argv[1]));
    const int nb = std::atoi(argv[2]), nh = std::atoi(argv[3]);
    const double zero_frac = std::atof(argv[4]);
    const int max_items = std::atoi(argv[5]);
    const int np = 4;
    std::mt19937 rng(seed);
    std::uniform_real_distribution<double> U(0.0, 1.0);
    std::vector<int> deck(52);
    for (int i = 0; i < 52; ++i) deck[i] = i;
    std::shuffle(deck.begin(), deck.end(), rng);
    int board[5];
    for (int i = 0; i < nb; ++i) board[i] = deck[i];
    const bool river = nb == 5;
    float bets[1] = {1.0f};
    int order[SS_MAX_PLAYERS] = {0, 1, 2, 3, 4, 5};
    BuiltTree bt;
    if (build_street_tree(board, nb, 300, 1000, bets, 1, np, order, river ? 1 : 0, river ? 0 : 1, 1, &bt) != SS_OK)
        return 3;
    // ranges: nh distinct non-board combos per player, U(0,1) weights
    std::vector<std::pair<int, int>> combos;
    for (int a = 0; a < 52; ++a)
        for (int b = a + 1; b < 52; ++b) {
            bool on = false;
            for (int i = 0; i < nb; ++i) on = on || board[i] == a || board[i] == b;
            if (!on) combos.push_back({a, b});
        }
    std::vector<int> hands[SS_MAX_PLAYERS];
    std::vector<float> wts[SS_MAX_PLAYERS];
    for (int p = 0; p < np; ++p) {
        std::shuffle(combos.begin(), combos.end(), rng);
        for (int h = 0; h < nh; ++h) {
            hands[p].push_back(combos[h].first);
            hands[p].push_back(combos[h].second);
            wts[p].push_back(static_cast<float>(U(rng)));
        }
    }
    std::vector<float> lv(static_cast<size_t>(bt.num_leaves) * np * nh);
    for (auto &x : lv) x = static_cast<float>(2.0 * U(rng) - 1.0);
    Problem pb{};
    pb.nodes = bt.nodes.data();
    pb.children = bt.children.data();
    pb.num_nodes = static_cast<int>(bt.nodes.size());
    pb.num_children_total = static_cast<int>(bt.children.size());
    pb.num_players = np;
    for (int p = 0; p < np; ++p) {
        pb.hands[p] = hands[p].data();
        pb.weights[p] = wts[p].data();
        pb.num_hands[p] = nh;
    }
    for (int i = 0; i < nb; ++i) pb.board[i] = board[i];
    pb.num_board = nb;
    pb.is_river = river ? 1 : 0;
    pb.starting_pot = 300;
    if (!river && bt.num_leaves > 0) {
        pb.leaf_values = lv.data();
        pb.num_leaves = bt.num_leaves;
    }
    Plan P;
    if (build_plan(pb, &P) != SS_OK) {
        std::fprintf(stderr, "%s\n", last_error());
        return 4;
    }
    const int HS = P.HS, rows = P.E + np;
    std::vector<float> reach(static_cast<size_t>(rows) * HS, 0.0f);
    for (int r = 0; r < rows; ++r)
        for (int h = 0; h < nh; ++h)
            reach[static_cast<size_t>(r) * HS + h] = U(rng) < zero_frac ? 0.0f : static_cast<float>(U(rng));
    auto card = [&](int p, int h, int k) { return P.hand_code[static_cast<size_t>(p) * HS + h] >> (8 * k) & 0xff; };
    auto blocked = [&](int p, int h) { return (P.hand_code[static_cast<size_t>(p) * HS + h] & 0x10000) != 0; };
    auto disjoint = [&](int p, int h, int q, int g) {
        return card(p, h, 0) != card(q, g, 0) && card(p, h, 0) != card(q, g, 1) && card(p, h, 1) != card(q, g, 0) &&
               card(p, h, 1) != card(q, g, 1);
    };

    double max_rel = 0.0;
    int items = 0, checked = 0, zero_bad = 0;
    Block blk(HS);
    Tables &t = blk.t;
    for (int trav = 0; trav < np; ++trav) {
        // --- folds / leaves with three counted opponents ---------------------------------
        const std::vector<TermItem> &cr = P.term[trav][TK_CR3];
        int seen = 0;
        for (size_t i = 0; i < cr.size() && seen < max_items; ++i) {
            const TermItem &I0 = cr[i];
            if (I0.follow) continue;
            ++seen;
            const int ng = I0.gextra + 1;
            Opp3<float> in{reach.data() + static_cast<size_t>(I0.opp_row[0]) * HS,
                           reach.data() + static_cast<size_t>(I0.opp_row[1]) * HS,
                           reach.data() + static_cast<size_t>(I0.opp_row[2]) * HS,
                           P.pair_idx.data() + static_cast<size_t>(I0.opp_player[0]) * 52 * 52,
                           P.pair_idx.data() + static_cast<size_t>(I0.opp_player[1]) * 52 * 52,
                           P.hand_code.data() + static_cast<size_t>(I0.opp_player[2]) * HS,
                           P.H[I0.opp_player[2]], HS, P.deck};
            for (int tid = 0; tid < kNt; ++tid) phase_gather(tid, kNt, in, t);
            for (int tid = 0; tid < kNt; ++tid) phase_rows(tid, kNt, t);
            for (int tid = 0; tid < kNt; ++tid) phase_product(tid, kNt, t);
            for (int tid = 0; tid < kNt; ++tid) phase_vectors(tid, kNt, in, t);
            for (int tid = 0; tid < kNt; ++tid) phase_scalars(tid, t);
            for (int h = 0; h < P.H[trav]; ++h) {
                const double m = cr3_hand_value_mass(P.hand_code[static_cast<size_t>(trav) * HS + h], P.deck, t);
                // enumeration: live, positive-reach, pairwise disjoint opponent hands avoiding the traverser
                const int o[3] = {I0.opp_player[0], I0.opp_player[1], I0.opp_player[2]};
                const float *rr[3] = {in.r1, in.r2, in.r3};
                double want = 0.0;
                for (int h1 = 0; h1 < P.H[o[0]]; ++h1) {
                    if (blocked(o[0], h1) || !(rr[0][h1] > 0.0f) || !disjoint(o[0], h1, trav, h)) continue;
                    for (int h2 = 0; h2 < P.H[o[1]]; ++h2) {
                        if (blocked(o[1], h2) || !(rr[1][h2] > 0.0f) || !disjoint(o[1], h2, trav, h) ||
                            !disjoint(o[1], h2, o[0], h1))
                            continue;
                        for (int h3 = 0; h3 < P.H[o[2]]; ++h3) {
                            if (blocked(o[2], h3) || !(rr[2][h3] > 0.0f) || !disjoint(o[2], h3, trav, h) ||
                                !disjoint(o[2], h3, o[0], h1) || !disjoint(o[2], h3, o[1], h2))
                                continue;
                            want += static_cast<double>(rr[0][h1]) * rr[1][h2] * rr[2][h3];
                        }
                    }
                }
                for (int g = 0; g < ng; ++g) {
                    const TermItem &Ig = (&I0)[g];
                    const double f = Ig.leaf_off >= 0 ? lv[static_cast<size_t>(Ig.leaf_off) + h] : Ig.payoff;
                    const double got = f * m, ref = f * want;
                    max_rel = std::max(max_rel, std::fabs(got - ref) / (1.0 + std::fabs(ref)));
                    if (ref == 0.0 && got != 0.0 && want == 0.0) ++zero_bad;
                    ++checked;
                }
            }
            items += ng;
        }
        // --- four-way showdowns -----------------------------------------------------------
        const std::vector<TermItem> &sd = P.term[trav][TK_SD3];
        for (size_t i = 0; i < sd.size() && static_cast<int>(i) < max_items; ++i) {
            const TermItem &I = sd[i];
            const int o1 = I.opp_player[0], o2 = I.opp_player[1], o3 = I.opp_player[2];
            Opp3<float> in{reach.data() + static_cast<size_t>(I.opp_row[0]) * HS,
                           reach.data() + static_cast<size_t>(I.opp_row[1]) * HS,
                           reach.data() + static_cast<size_t>(I.opp_row[2]) * HS,
                           P.pair_idx.data() + static_cast<size_t>(o1) * 52 * 52,
                           P.pair_idx.data() + static_cast<size_t>(o2) * 52 * 52,
                           P.hand_code.data() + static_cast<size_t>(o3) * HS, P.H[o3], HS, P.deck};
            const int *posA = P.sd_pos.data() + static_cast<size_t>(o1) * HS;
            const int *posB = P.sd_pos.data() + static_cast<size_t>(o2) * HS;
            std::vector<double> out(static_cast<size_t>(HS), -1e300);
            auto build = [&](int lo1, int hi1, int lo2, int hi2) {
                for (int tid = 0; tid < kNt; ++tid) phase_gather_cls(tid, kNt, in, t, posA, lo1, hi1, posB, lo2, hi2);
                for (int tid = 0; tid < kNt; ++tid) phase_rows(tid, kNt, t);
                for (int tid = 0; tid < kNt; ++tid) phase_product(tid, kNt, t);
                for (int tid = 0; tid < kNt; ++tid) phase_vectors(tid, kNt, in, t, false);
                for (int tid = 0; tid < kNt; ++tid) phase_scalars(tid, t);
            };
            const int nc = P.ncomb;
            for (int ch = 0; ch * kNt < nc; ++ch) {
                const int q0 = ch * kNt, qend = std::min(q0 + kNt, nc);
                std::vector<Sd3Thread> st(kNt);
                for (int tid = 0; tid < kNt; ++tid)
                    sd3_thread_init(q0 + tid, qend, P.pos_hand.data() + static_cast<size_t>(trav) * nc,
                                    P.hand_code.data() + static_cast<size_t>(trav) * HS, P.sd_combo.data(), st[tid]);
                compact_third(0, in, t, P.sd_pos.data() + static_cast<size_t>(o3) * HS, blk.p3.data());
                build(0, 1 << 30, 0, 1 << 30);
                for (int tid = 0; tid < kNt; ++tid) sd3_thread_total(st[tid], t, blk.p3.data());
                for (int g = q0; g < qend;) {
                    const int lo = P.sd_combo[g].lo, hi = P.sd_combo[g].hi;
                    bool any = false;
                    for (int tid = 0; tid < kNt; ++tid) any = any || (st[tid].h >= 0 && st[tid].glo == lo);
                    if (any)
                        for (int pr = 0; pr < 4; ++pr) {
                            int lo1, hi1, lo2, hi2;
                            sd3_pair_bounds(pr, lo, hi, &lo1, &hi1, &lo2, &hi2);
                            build(lo1, hi1, lo2, hi2);
                            for (int tid = 0; tid < kNt; ++tid)
                                if (st[tid].h >= 0 && st[tid].glo == lo)
                                    sd3_thread_pair(st[tid], t, blk.p3.data(), pr, lo, hi);
                        }
                    g = hi;
                }
                for (int tid = 0; tid < kNt; ++tid)
                    if (st[tid].h >= 0) out[static_cast<size_t>(st[tid].h)] = sd3_thread_value(st[tid], I.pot, I.bet);
            }
            const unsigned *S = P.strength.data();
            const double cw = static_cast<double>(I.pot - I.bet), c2 = static_cast<double>(I.pot / 2.0f - I.bet);
            const double c3 = static_cast<double>(I.pot / 3.0f - I.bet), c4 = static_cast<double>(I.pot / 4.0f - I.bet);
            const double cl = -static_cast<double>(I.bet);
            for (int h = 0; h < P.H[trav]; ++h) {
                const unsigned s0 = S[static_cast<size_t>(trav) * HS + h];
                if (s0 == 0) continue;   // no rank position: the first block writes 0
                const int o[3] = {o1, o2, o3};
                const float *rr[3] = {in.r1, in.r2, in.r3};
                double want = 0.0, scale = 0.0;
                long long tuples = 0;
                for (int h1 = 0; h1 < P.H[o1]; ++h1) {
                    const unsigned s1 = S[static_cast<size_t>(o1) * HS + h1];
                    if (s1 == 0 || !(rr[0][h1] > 0.0f) || !disjoint(o1, h1, trav, h)) continue;
                    for (int h2 = 0; h2 < P.H[o2]; ++h2) {
                        const unsigned s2 = S[static_cast<size_t>(o2) * HS + h2];
                        if (s2 == 0 || !(rr[1][h2] > 0.0f) || !disjoint(o2, h2, trav, h) || !disjoint(o2, h2, o1, h1))
                            continue;
                        for (int h3 = 0; h3 < P.H[o3]; ++h3) {
                            const unsigned s3 = S[static_cast<size_t>(o3) * HS + h3];
                            if (s3 == 0 || !(rr[2][h3] > 0.0f) || !disjoint(o3, h3, trav, h) ||
                                !disjoint(o3, h3, o1, h1) || !disjoint(o3, h3, o2, h2))
                                continue;
                            const double m = static_cast<double>(rr[0][h1]) * rr[1][h2] * rr[2][h3];
                            const unsigned best = std::max(std::max(s1, s2), s3);
                            double coef = cl;
                            if (s0 >= best) {
                                const int wins = 1 + (s1 == s0) + (s2 == s0) + (s3 == s0);
                                coef = wins == 1 ? cw : wins == 2 ? c2 : wins == 3 ? c3 : c4;
                            }
                            want += coef * m;
                            scale += std::fabs(coef * m);
                            ++tuples;
                        }
                    }
                }
                const double got = out[static_cast<size_t>(h)];
                max_rel = std::max(max_rel, std::fabs(got - want) / (1.0 + scale));
                if (tuples == 0 && got != 0.0) ++zero_bad;
                ++checked;
            }
            ++items;
        }
    }
    std::printf("{\"items\": %d, \"hands\": %d, \"max_rel_err\": %.3e, \"zero_bad\": %d, \"cr3\": %zu, \"sd3\": %zu}\n",
                items, checked, max_rel, zero_bad, P.term[0][TK_CR3].size(), P.term[0][TK_SD3].size());
    return 0;
}
