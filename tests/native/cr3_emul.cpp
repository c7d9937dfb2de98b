// Runs the three-counted-opponent block phases (poker-solver_b200/csrc/
// ss_cr3.cuh) on the host -- each phase over 256 emulated threads, phases
// in kernel order -- and compares every traverser hand with brute-force
// enumeration of the disjoint opponent tuples, for tests/test_cr3_host.py.
//   cr3_emul <seed> <deck> <hands per player> <zero fraction> [zero player]
// Hands are random distinct pairs over the dense deck 0..deck-1; about a
// tenth of every range touches the board (dense index 63, as the planner
// codes it); weights U(0,1) with the given fraction zeroed (all of them for
// the zero player, if given).  Prints JSON: the largest relative mass error,
// count mismatches, and whether every hand without a positive tuple gets
// exactly 0 under the kernel's rule.
#include "ss_cr3.cuh"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <utility>
#include <vector>

using namespace ssb::cr3;

int main(int argc, char **argv) {
    if (argc < 5) return 2;
    const unsigned seed = static_cast<unsigned>(std::atoi(argv[1]));
    const int deck = std::atoi(argv[2]), nh = std::atoi(argv[3]);
    const double zero_frac = std::atof(argv[4]);
    const int zero_player = argc > 5 ? std::atoi(argv[5]) : -1;
    if (deck < 4 || deck > 49 || nh < 1) return 2;
    std::mt19937 rng(seed);
    std::uniform_real_distribution<double> U(0.0, 1.0);
    const int HS = ((nh + 31) / 32) * 32;
    // players 0..2: the counted opponents; player 3: the traverser
    std::vector<std::vector<int>> code(4, std::vector<int>(HS, 0));
    std::vector<std::vector<float>> reach(3, std::vector<float>(HS + 4, 0.0f));
    for (int p = 0; p < 4; ++p) {
        std::vector<std::pair<int, int>> all;
        for (int a = 0; a < deck; ++a)
            for (int b = a + 1; b < deck; ++b) all.push_back({a, b});
        std::shuffle(all.begin(), all.end(), rng);
        for (int h = 0; h < nh; ++h) {
            int a = all[h % all.size()].first, b = all[h % all.size()].second;
            int blocked = 0;
            if (U(rng) < 0.1) {   // one card on the board
                if (U(rng) < 0.5) a = 63; else b = 63;
                blocked = 1;
            }
            code[p][h] = (blocked << 16) | (a << 20) | (b << 26);
            if (p < 3) {
                const bool zero = p == zero_player || U(rng) < zero_frac;
                reach[p][h] = zero ? 0.0f : static_cast<float>(U(rng));
            }
        }
    }
    // pair tables of the two matrix opponents, as the planner builds them
    std::vector<int> pair[2];
    for (int p = 0; p < 2; ++p) {
        pair[p].assign(52 * 52, HS);
        for (int h = 0; h < nh; ++h) {
            if (code[p][h] & 0x10000) continue;
            const int a = (code[p][h] >> 20) & 63, b = (code[p][h] >> 26) & 63;
            pair[p][a * 52 + b] = h;
            pair[p][b * 52 + a] = h;
        }
    }
    std::vector<double> A(kS * kS), B(kS * kS), P(kS * kS), PT(kS * kS), uA(kS), uB(kS), w(kS), d(kS), sc(8), r3(HS);
    std::vector<int> iuA(kS), iuB(kS), iw(kS), id(kS);
    std::vector<unsigned long long> mA(kS), mB(kS);
    std::vector<long long> isc(8);
    std::vector<unsigned short> xy(HS);
    Tables t{A.data(), B.data(), P.data(), PT.data(), uA.data(), uB.data(), w.data(), d.data(),
             iuA.data(), iuB.data(), iw.data(), id.data(), mA.data(), mB.data(), r3.data(), xy.data(),
             sc.data(), isc.data()};
    Opp3<float> in{reach[0].data(), reach[1].data(), reach[2].data(), pair[0].data(), pair[1].data(),
                   code[2].data(), nh, HS, deck};
    const int nt = 256;
    for (int tid = 0; tid < nt; ++tid) phase_gather(tid, nt, in, t);
    for (int tid = 0; tid < nt; ++tid) phase_rows(tid, nt, t);
    for (int tid = 0; tid < nt; ++tid) phase_product_tiled(tid, nt, t);
    for (int tid = 0; tid < nt; ++tid) phase_vectors(tid, nt, in, t);
    for (int tid = 0; tid < nt; ++tid) phase_scalars(tid, t);
    const double zb = zero_bound(t);

    auto cards = [&](int p, int h, int *c0, int *c1) {
        *c0 = (code[p][h] >> 20) & 63;
        *c1 = (code[p][h] >> 26) & 63;
    };
    double max_rel = 0.0;
    int mismatches = 0, zero_hands = 0, zero_bad = 0;
    for (int h = 0; h < nh; ++h) {
        int ta, tb;
        cards(3, h, &ta, &tb);
        // brute force: every tuple of live, positive-reach, pairwise disjoint hands avoiding the traverser
        double want = 0.0;
        long long cnt = 0;
        for (int o1 = 0; o1 < nh; ++o1) {
            if ((code[0][o1] & 0x10000) || !(reach[0][o1] > 0.0f)) continue;
            int a1, b1;
            cards(0, o1, &a1, &b1);
            if (a1 == ta || a1 == tb || b1 == ta || b1 == tb) continue;
            for (int o2 = 0; o2 < nh; ++o2) {
                if ((code[1][o2] & 0x10000) || !(reach[1][o2] > 0.0f)) continue;
                int a2, b2;
                cards(1, o2, &a2, &b2);
                if (a2 == ta || a2 == tb || b2 == ta || b2 == tb || a2 == a1 || a2 == b1 || b2 == a1 || b2 == b1)
                    continue;
                for (int o3 = 0; o3 < nh; ++o3) {
                    if ((code[2][o3] & 0x10000) || !(reach[2][o3] > 0.0f)) continue;
                    int a3, b3;
                    cards(2, o3, &a3, &b3);
                    if (a3 == ta || a3 == tb || b3 == ta || b3 == tb || a3 == a1 || a3 == b1 || b3 == a1 ||
                        b3 == b1 || a3 == a2 || a3 == b2 || b3 == a2 || b3 == b2)
                        continue;
                    want += static_cast<double>(reach[0][o1]) * reach[1][o2] * reach[2][o3];
                    ++cnt;
                }
            }
        }
        const int a = ta >= deck ? deck : ta, b = tb >= deck ? deck : tb;
        double m = hand_mass(a, b, t);
        const long long c = hand_count(a, b, t);
        if (c != cnt) ++mismatches;
        const double rel = std::fabs(m - want) / (1.0 + std::fabs(want));
        max_rel = std::max(max_rel, rel);
        if (std::fabs(m) <= zb && hand_count(a, b, t) == 0) m = 0.0;   // the kernel's rule
        if (cnt == 0) {
            ++zero_hands;
            if (m != 0.0) ++zero_bad;
        }
    }
    std::printf("{\"hands\": %d, \"max_rel_err\": %.3e, \"count_mismatches\": %d, \"zero_hands\": %d, "
                "\"zero_bad\": %d, \"o3_entries\": %lld}\n",
                nh, max_rel, mismatches, zero_hands, zero_bad, t.isc[4]);
    return 0;
}
