// Checks the sparse four-way showdown steps of poker-solver_b200/csrc/
// ss_cr3.cuh on the host, for tests/test_cr3_host.py:
//  * add_hands: tables grown hand by hand along the rank positions equal a
//    direct build of the weaker parts at every tie group (FP64 fields to
//    rounding, counts and masks exactly);
//  * e_pair_slice: the pairs with a tying part (EL, LE, EE) evaluated from
//    the weaker parts' tables and the tying hands' lists equal the class
//    masses of a direct build of the pair, and their tuple counts equal
//    brute-force enumeration.
//   sd3inc_emul <seed> <deck> <hands per player> <zero fraction> <rank levels>
// Rank positions are abstract levels as in sd3_emul.  Prints JSON: the
// largest relative error of the tables and of the class masses, and the
// number of count mismatches.
#include "ss_cr3.cuh"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <utility>
#include <vector>

using namespace ssb::cr3;

struct TableStore {
    std::vector<double> A, B, P, PT, uA, uB, w, d, sc, r3;
    std::vector<int> iuA, iuB, iw, id;
    std::vector<unsigned long long> mA, mB;
    std::vector<long long> isc;
    std::vector<unsigned short> xy;
    Tables t;
    explicit TableStore(int HS)
        : A(kS * kS), B(kS * kS), P(kS * kS), PT(kS * kS), uA(kS), uB(kS), w(kS), d(kS), sc(8), r3(HS),
          iuA(kS), iuB(kS), iw(kS), id(kS), mA(kS), mB(kS), isc(8), xy(HS) {
        t = Tables{A.data(), B.data(), P.data(), PT.data(), uA.data(), uB.data(), w.data(), d.data(),
                   iuA.data(), iuB.data(), iw.data(), id.data(), mA.data(), mB.data(), r3.data(), xy.data(),
                   sc.data(), isc.data()};
    }
};

static double rel(double a, double b) { return std::fabs(a - b) / (1.0 + std::fabs(b)); }

// largest relative difference of the FP64 fields; integer fields must match
static double compare(const TableStore &x, const TableStore &y, int *bad) {
    double m = 0.0;
    for (int i = 0; i < kS * kS; ++i) {
        m = std::max(m, rel(x.A[i], y.A[i]));
        m = std::max(m, rel(x.B[i], y.B[i]));
        m = std::max(m, rel(x.P[i], y.P[i]));
        m = std::max(m, rel(x.PT[i], y.PT[i]));
    }
    for (int c = 0; c < kS; ++c) {
        m = std::max(m, rel(x.uA[c], y.uA[c]));
        m = std::max(m, rel(x.uB[c], y.uB[c]));
        m = std::max(m, rel(x.w[c], y.w[c]));
        m = std::max(m, rel(x.d[c], y.d[c]));
        if (x.iuA[c] != y.iuA[c] || x.iuB[c] != y.iuB[c] || x.iw[c] != y.iw[c] || x.id[c] != y.id[c] ||
            x.mA[c] != y.mA[c] || x.mB[c] != y.mB[c])
            ++*bad;
    }
    for (int i = 0; i < 4; ++i) {
        m = std::max(m, rel(x.sc[i], y.sc[i]));
        if (x.isc[i] != y.isc[i]) ++*bad;
    }
    return m;
}

int main(int argc, char **argv) {
    if (argc != 6) return 2;
    const unsigned seed = static_cast<unsigned>(std::atoi(argv[1]));
    const int deck = std::atoi(argv[2]), nh = std::atoi(argv[3]);
    const double zero_frac = std::atof(argv[4]);
    const int levels = std::atoi(argv[5]);
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
            const int a = all[h % all.size()].first, b = all[h % all.size()].second;
            code[p][h] = (a << 20) | (b << 26);
            pos[p][h] = static_cast<int>(rng() % static_cast<unsigned>(levels));
            if (p < 3) reach[p][h] = U(rng) < zero_frac ? 0.0f : static_cast<float>(U(rng));
        }
    }
    std::vector<int> pair[2];
    for (int p = 0; p < 2; ++p) {
        pair[p].assign(52 * 52, HS);
        for (int h = 0; h < nh; ++h) {
            const int a = (code[p][h] >> 20) & 63, b = (code[p][h] >> 26) & 63;
            pair[p][a * 52 + b] = h;
            pair[p][b * 52 + a] = h;
        }
    }
    TableStore inc(HS), dir(HS);
    std::vector<int> p3(HS);
    Opp3<float> in{reach[0].data(), reach[1].data(), reach[2].data(), pair[0].data(), pair[1].data(),
                   code[2].data(), nh, HS, deck};
    const int nt = 256;
    compact_third(0, in, inc.t, pos[2].data(), p3.data());
    compact_third(0, in, dir.t, pos[2].data(), p3.data());
    auto build = [&](Tables &t, int lo1, int hi1, int lo2, int hi2) {
        for (int tid = 0; tid < nt; ++tid) phase_gather_cls(tid, nt, in, t, pos[0].data(), lo1, hi1, pos[1].data(), lo2, hi2);
        for (int tid = 0; tid < nt; ++tid) phase_rows(tid, nt, t);
        for (int tid = 0; tid < nt; ++tid) phase_product_tiled(tid, nt, t);
        for (int tid = 0; tid < nt; ++tid) phase_vectors(tid, nt, in, t, false);
        for (int tid = 0; tid < nt; ++tid) phase_scalars(tid, t);
    };
    auto elist = [&](int p, int v) {
        std::vector<EHand> L;
        for (int h = 0; h < nh; ++h)
            if (pos[p][h] == v && reach[p][h] > 0.0f)
                L.push_back(EHand{static_cast<double>(reach[p][h]), (code[p][h] >> 20) & 63, (code[p][h] >> 26) & 63});
        return L;
    };
    double max_tab = 0.0, max_rel = 0.0;
    int bad = 0, checked = 0;
    build(inc.t, 0, 0, 0, 0);   // empty weaker parts
    for (int v = 0; v < levels; ++v) {
        // the grown tables against a direct build of the weaker parts [0, v)
        build(dir.t, 0, v, 0, v);
        max_tab = std::max(max_tab, compare(inc, dir, &bad));
        const std::vector<EHand> E1 = elist(0, v), E2 = elist(1, v);
        for (int h = 0; h < nh; ++h) {
            if (pos[3][h] != v) continue;
            const int a = (code[3][h] >> 20) & 63, b = (code[3][h] >> 26) & 63;
            for (int pr = 1; pr < 4; ++pr) {
                // the direct evaluation from the grown tables, sliced as a block
                // spreads it over lanes, against the pair's own tables
                double so[2] = {0.0, 0.0};
                long long sn[2] = {0, 0};
                for (int k0 = 0; k0 < 64; ++k0) {
                    double o[2];
                    long long n[2];
                    e_pair_slice(pr, a, b, inc.t, E1.data(), static_cast<int>(E1.size()), E2.data(),
                                 static_cast<int>(E2.size()), p3.data(), v, v + 1, k0, 64, o, n);
                    for (int c = 0; c < 2; ++c) {
                        so[c] += o[c];
                        sn[c] += n[c];
                    }
                }
                TableStore pt(HS);
                compact_third(0, in, pt.t, pos[2].data(), p3.data());
                build(pt.t, (pr & 1) ? v : 0, (pr & 1) ? v + 1 : v, (pr & 2) ? v : 0, (pr & 2) ? v + 1 : v);
                double o3[3];
                long long c3[3];
                hand_mass_cls(a, b, pt.t, p3.data(), v, v + 1, o3, c3, true);
                for (int c = 0; c < 2; ++c) {
                    if (sn[c] != c3[c]) ++bad;
                    if (sn[c] == 0 && so[c] != 0.0) ++bad;
                    max_rel = std::max(max_rel, std::fabs(so[c] - o3[c]) / (1.0 + std::fabs(o3[c])));
                }
            }
            ++checked;
        }
        // grow the tables by this level's hands: the first opponent's, then the second's
        for (int tid = 0; tid < nt; ++tid) add_hands(tid, nt, inc.t, 0, E1.data(), static_cast<int>(E1.size()));
        for (int tid = 0; tid < nt; ++tid) add_hands(tid, nt, inc.t, 1, E2.data(), static_cast<int>(E2.size()));
    }
    std::printf("{\"hands\": %d, \"max_table_err\": %.3e, \"max_rel_err\": %.3e, \"bad\": %d}\n", checked, max_tab,
                max_rel, bad);
    return 0;
}
