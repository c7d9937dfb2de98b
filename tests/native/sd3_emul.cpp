// Runs the four-way showdown class masses of poker-solver_b200/csrc/
// ss_cr3.cuh on the host -- for each traverser hand the tables of the five
// matrix pairs (all, and the first two opponents' weaker / tying parts)
// built phase by phase over 256 emulated threads -- and compares every
// class mass and the showdown value with brute-force enumeration of the
// disjoint opponent tuples (the reference's rule, street_solve.cu:936-1002),
// for tests/test_cr3_host.py.
//   sd3_emul <seed> <deck> <hands per player> <zero fraction> <rank levels> <pot> <bet>
// Rank positions are abstract: each live hand gets a level in [0, levels)
// (few levels: many ties); a hand holding a board card has none.  Prints
// JSON: the largest relative error of the class masses and values, and the
// number of classes without a tuple whose mass is not exactly 0.
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
    if (argc != 8) return 2;
    const unsigned seed = static_cast<unsigned>(std::atoi(argv[1]));
    const int deck = std::atoi(argv[2]), nh = std::atoi(argv[3]);
    const double zero_frac = std::atof(argv[4]);
    const int levels = std::atoi(argv[5]);
    const float pot = static_cast<float>(std::atof(argv[6])), bet = static_cast<float>(std::atof(argv[7]));
    if (deck < 4 || deck > 49 || nh < 1 || levels < 1) return 2;
    std::mt19937 rng(seed);
    std::uniform_real_distribution<double> U(0.0, 1.0);
    const int HS = ((nh + 31) / 32) * 32;
    // players 0..2: the live opponents; player 3: the traverser
    std::vector<std::vector<int>> code(4, std::vector<int>(HS, 0)), pos(4, std::vector<int>(HS, -1));
    std::vector<std::vector<float>> reach(3, std::vector<float>(HS + 4, 0.0f));
    for (int p = 0; p < 4; ++p) {
        std::vector<std::pair<int, int>> all;
        for (int a = 0; a < deck; ++a)
            for (int b = a + 1; b < deck; ++b) all.push_back({a, b});
        std::shuffle(all.begin(), all.end(), rng);
        for (int h = 0; h < nh; ++h) {
            int a = all[h % all.size()].first, b = all[h % all.size()].second;
            int blocked = 0;
            if (U(rng) < 0.1) {
                if (U(rng) < 0.5) a = 63; else b = 63;
                blocked = 1;
            }
            code[p][h] = (blocked << 16) | (a << 20) | (b << 26);
            pos[p][h] = blocked ? -1 : static_cast<int>(rng() % static_cast<unsigned>(levels));
            if (p < 3) reach[p][h] = U(rng) < zero_frac ? 0.0f : static_cast<float>(U(rng));
        }
    }
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
    std::vector<int> iuA(kS), iuB(kS), iw(kS), id(kS), p3(HS);
    std::vector<unsigned long long> mA(kS), mB(kS);
    std::vector<long long> isc(8);
    std::vector<unsigned short> xy(HS);
    Tables t{A.data(), B.data(), P.data(), PT.data(), uA.data(), uB.data(), w.data(), d.data(),
             iuA.data(), iuB.data(), iw.data(), id.data(), mA.data(), mB.data(), r3.data(), xy.data(),
             sc.data(), isc.data()};
    Opp3<float> in{reach[0].data(), reach[1].data(), reach[2].data(), pair[0].data(), pair[1].data(),
                   code[2].data(), nh, HS, deck};
    const int nt = 256, BIG = 1 << 30;
    compact_third(0, in, t, pos[2].data(), p3.data());
    auto build = [&](int lo1, int hi1, int lo2, int hi2) {
        for (int tid = 0; tid < nt; ++tid) phase_gather_cls(tid, nt, in, t, pos[0].data(), lo1, hi1, pos[1].data(), lo2, hi2);
        for (int tid = 0; tid < nt; ++tid) phase_rows(tid, nt, t);
        for (int tid = 0; tid < nt; ++tid) phase_product_tiled(tid, nt, t);
        for (int tid = 0; tid < nt; ++tid) phase_vectors(tid, nt, in, t, false);
        for (int tid = 0; tid < nt; ++tid) phase_scalars(tid, t);
    };
    const Sd3Coef k{static_cast<double>(pot - bet), static_cast<double>(pot / 2.0f - bet),
                    static_cast<double>(pot / 3.0f - bet), static_cast<double>(pot / 4.0f - bet),
                    -static_cast<double>(bet)};
    auto cards = [&](int p, int h, int *c0, int *c1) {
        *c0 = (code[p][h] >> 20) & 63;
        *c1 = (code[p][h] >> 26) & 63;
    };
    double max_rel = 0.0;
    int zero_bad = 0, checked = 0, empty_classes = 0;
    for (int h = 0; h < nh; ++h) {
        const int v = pos[3][h];
        if (v < 0) continue;
        int ta, tb;
        cards(3, h, &ta, &tb);
        const int a = ta, b = tb;   // live traverser hands hold no board card
        // brute force: per pair class (first, second opponent) x third's class, and the total
        double bm[4][2] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}}, btot = 0.0, bval = 0.0;
        long long bc[4][2] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}}, bct = 0;
        for (int o1 = 0; o1 < nh; ++o1) {
            if (pos[0][o1] < 0 || !(reach[0][o1] > 0.0f)) continue;
            int a1, b1;
            cards(0, o1, &a1, &b1);
            if (a1 == ta || a1 == tb || b1 == ta || b1 == tb) continue;
            for (int o2 = 0; o2 < nh; ++o2) {
                if (pos[1][o2] < 0 || !(reach[1][o2] > 0.0f)) continue;
                int a2, b2;
                cards(1, o2, &a2, &b2);
                if (a2 == ta || a2 == tb || b2 == ta || b2 == tb || a2 == a1 || a2 == b1 || b2 == a1 || b2 == b1)
                    continue;
                for (int o3 = 0; o3 < nh; ++o3) {
                    if (pos[2][o3] < 0 || !(reach[2][o3] > 0.0f)) continue;
                    int a3, b3;
                    cards(2, o3, &a3, &b3);
                    if (a3 == ta || a3 == tb || b3 == ta || b3 == tb || a3 == a1 || a3 == b1 || b3 == a1 ||
                        b3 == b1 || a3 == a2 || a3 == b2 || b3 == a2 || b3 == b2)
                        continue;
                    const double m = static_cast<double>(reach[0][o1]) * reach[1][o2] * reach[2][o3];
                    btot += m;
                    ++bct;
                    const int s1 = pos[0][o1], s2 = pos[1][o2], s3 = pos[2][o3];
                    if (s1 > v || s2 > v || s3 > v) {
                        bval += k.loss * m;
                        continue;
                    }
                    const int winners = 1 + (s1 == v) + (s2 == v) + (s3 == v);
                    bval += (winners == 1 ? k.win : winners == 2 ? k.two : winners == 3 ? k.three : k.four) * m;
                    const int pr = (s1 == v ? 1 : 0) + (s2 == v ? 2 : 0);   // LL, EL, LE, EE
                    bm[pr][s3 == v ? 1 : 0] += m;
                    ++bc[pr][s3 == v ? 1 : 0];
                }
            }
        }
        // the closed form, as the kernel evaluates it for this hand's group [v, v + 1)
        double m[4][2], tot3[3];
        long long cnt[3];
        build(0, BIG, 0, BIG);
        hand_mass_cls(a, b, t, p3.data(), v, v + 1, tot3, cnt, true);
        double total = tot3[2];
        if (std::fabs(total) <= zero_bound(t) && cnt[2] == 0) total = 0.0;
        const int r1[4][2] = {{0, v}, {v, v + 1}, {0, v}, {v, v + 1}};
        const int r2[4][2] = {{0, v}, {0, v}, {v, v + 1}, {v, v + 1}};
        for (int pr = 0; pr < 4; ++pr) {
            build(r1[pr][0], r1[pr][1], r2[pr][0], r2[pr][1]);
            double o[3];
            long long c[3];
            hand_mass_cls(a, b, t, p3.data(), v, v + 1, o, c, true);
            // the kernel's split of the same sums: per warps of 32 lanes, each
            // lane every (per * 32)-th entry of the third opponent's list
            for (int per = 1; per <= 8; per *= 2) {
                double so[2] = {0.0, 0.0};
                long long sc[2] = {0, 0};
                for (int k0 = 0; k0 < per * 32; ++k0) {
                    double po[2], unused_o[2];
                    long long pc[2], unused_c[2];
                    hand_mass_cls_slice(a, b, t, p3.data(), v, v + 1, k0, per * 32, po, unused_c, false);
                    hand_mass_cls_slice(a, b, t, p3.data(), v, v + 1, k0, per * 32, unused_o, pc, true);
                    for (int cl = 0; cl < 2; ++cl) {
                        so[cl] += po[cl];
                        sc[cl] += pc[cl];
                    }
                }
                for (int cl = 0; cl < 2; ++cl) {
                    if (sc[cl] != c[cl]) ++zero_bad;
                    max_rel = std::max(max_rel, std::fabs(so[cl] - o[cl]) / (1.0 + std::fabs(o[cl])));
                }
            }
            const double zb = zero_bound(t);
            for (int cl = 0; cl < 2; ++cl) {
                m[pr][cl] = (std::fabs(o[cl]) <= zb && c[cl] == 0) ? 0.0 : o[cl];
                if (c[cl] != bc[pr][cl]) ++zero_bad;   // the count must be exact
                if (bc[pr][cl] == 0) {
                    ++empty_classes;
                    if (m[pr][cl] != 0.0) ++zero_bad;
                }
                max_rel = std::max(max_rel, std::fabs(m[pr][cl] - bm[pr][cl]) / (1.0 + std::fabs(bm[pr][cl])));
            }
        }
        if (cnt[2] != bct) ++zero_bad;
        const double val = sd3_value(m, total, k);
        max_rel = std::max(max_rel, std::fabs(total - btot) / (1.0 + std::fabs(btot)));
        max_rel = std::max(max_rel, std::fabs(val - bval) / (1.0 + std::fabs(bval) + std::fabs(k.loss * btot)));
        if (bct == 0 && val != 0.0) ++zero_bad;
        ++checked;
    }
    std::printf("{\"hands\": %d, \"max_rel_err\": %.3e, \"zero_bad\": %d, \"empty_classes\": %d}\n", checked,
                max_rel, zero_bad, empty_classes);
    return 0;
}
