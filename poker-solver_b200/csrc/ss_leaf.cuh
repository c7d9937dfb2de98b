// ss_leaf.cuh -- continuation-value producer, per-element arithmetic.
//
// Five phases, each a function of one flat element index so that a kernel
// is a grid-stride loop over it (ss_leaf.cu):
//   strength  (runout, player, hand)  7-card strength, 0 if a board card blocks the hand
//   digest    (opponent tuple)        union card mask, best strength, how many hold it
//   ratio     (runout, player, hand)  share of the tuples the hand beats
//   equity    (player, hand)          mean of the ratios over the runouts
//   value     (row, player, hand)     bias-adjusted value at the row's leaf pot
// The FP64 arithmetic follows the reference's Python expressions one
// operation at a time, rounded to nearest: the device form uses the _rn
// intrinsics so that no multiply-add is contracted, which keeps every value
// bit-identical to the reference module (python/leaf_values.py:91-121,
// 573-691, 768-814).
#pragma once

#include "ss_rank.cuh"

#include <cstdint>

namespace ssb {
namespace leaf {

struct Digest {
    unsigned long long mask;   // cards the opponents hold; all ones if two of them share a card
    unsigned best;             // the opponents' best strength
    unsigned nbest;            // how many opponents hold it
};

struct Ctx {
    int np, mh, nr, per, num_leaves;
    const int *nh;                 // [np]
    const int *hand_cards;         // [np][mh][2]
    const int *board5;             // [nr][5]
    const int *tuple_off;          // [nr*np + 1]
    const int *tuple_owner;        // [tuples]
    const uint16_t *tuple_hand;    // [tuples][np-1]
    const double *row_pot;         // [num_leaves]
    const unsigned char *row_set;  // [num_leaves]
    unsigned *strength;            // [nr][np][mh]
    Digest *digest;                // [tuples]
    double *ratio;                 // [nr][np][mh]; -1 where the runout does not count for the hand
    double *equity;                // [np][mh]
    float *values;                 // rows row0 .. of [rows][np][mh]
};

SSB_HD double dmul(double a, double b) {
#if defined(__CUDA_ARCH__)
    return __dmul_rn(a, b);
#else
    return a * b;
#endif
}
SSB_HD double dadd(double a, double b) {
#if defined(__CUDA_ARCH__)
    return __dadd_rn(a, b);
#else
    return a + b;
#endif
}
SSB_HD double dsub(double a, double b) {
#if defined(__CUDA_ARCH__)
    return __dsub_rn(a, b);
#else
    return a - b;
#endif
}
SSB_HD double ddiv(double a, double b) {
#if defined(__CUDA_ARCH__)
    return __ddiv_rn(a, b);
#else
    return a / b;
#endif
}

// python/leaf_values.py:91-121 with BIAS_FOLD_PROB / BIAS_POT_FACTOR (:84, :88)
SSB_HD double biased_value(double equity, double pot, int s_self, int s_opp) {
    const double fold = s_opp == 1 ? 0.35 : 0.0;
    const double pf_self = s_self == 1 ? 0.7 : (s_self == 3 ? 1.4 : 1.0);
    const double pf_opp = s_opp == 1 ? 0.7 : (s_opp == 3 ? 1.4 : 1.0);
    const double showdown_pot = dmul(pot, dmul(pf_self, pf_opp));
    const double fold_payoff = dmul(0.5, pot);
    const double showdown_payoff = dmul(dsub(equity, 0.5), showdown_pot);
    return dadd(dmul(fold, fold_payoff), dmul(dsub(1.0, fold), showdown_payoff));
}

// the opponents' profile seen by player p under continuation profile
// `combo` (python/leaf_values.py:800-808): the other player's for two
// players, else the mean of the others' rounded half to even (Python's
// round), which for these small integers is exact in integer arithmetic
SSB_HD int opponent_profile(int combo, int p, int np) {
    if (np == 2) return (combo >> (2 * (1 - p))) & 3;
    int sum = 0;
    for (int q = 0; q < np; ++q)
        if (q != p) sum += (combo >> (2 * q)) & 3;
    const int d = np - 1, fl = sum / d, rem = sum % d;
    const int r = 2 * rem > d ? fl + 1 : (2 * rem == d ? fl + (fl & 1) : fl);
    return r < 0 ? 0 : (r > 3 ? 3 : r);
}

SSB_HD void strength_at(long i, const Ctx &c) {
    const int h = static_cast<int>(i % c.mh);
    const int p = static_cast<int>((i / c.mh) % c.np);
    const long r = i / (static_cast<long>(c.mh) * c.np);
    unsigned s = 0u;
    if (h < c.nh[p]) {
        const int *hc = c.hand_cards + (static_cast<long>(p) * c.mh + h) * 2;
        const int *b = c.board5 + r * 5;
        int cards[7] = {b[0], b[1], b[2], b[3], b[4], hc[0], hc[1]};
        bool blocked = false;
        for (int k = 0; k < 5; ++k) blocked = blocked || b[k] == hc[0] || b[k] == hc[1];
        if (!blocked) s = rank7(cards);
    }
    c.strength[i] = s;
}

// python/leaf_values.py:633-675 for everything that does not depend on the hero hand
SSB_HD void digest_at(long t, const Ctx &c) {
    const int owner = c.tuple_owner[t];
    const int r = owner / c.np, hero = owner % c.np;
    const uint16_t *hands = c.tuple_hand + t * (c.np - 1);
    unsigned long long mask = 0ull;
    bool clash = false;
    unsigned best = 0u, nbest = 0u;
    for (int k = 0; k < c.np - 1; ++k) {
        const int q = k < hero ? k : k + 1;
        const int h = hands[k];
        const int *hc = c.hand_cards + (static_cast<long>(q) * c.mh + h) * 2;
        const unsigned long long bits = (1ull << hc[0]) | (1ull << hc[1]);
        clash = clash || (mask & bits) != 0ull;
        mask |= bits;
        const unsigned s = c.strength[(static_cast<long>(r) * c.np + q) * c.mh + h];
        if (s > best) {
            best = s;
            nbest = 1u;
        } else if (s == best) {
            ++nbest;
        }
    }
    Digest d;
    d.mask = clash ? ~0ull : mask;
    d.best = best;
    d.nbest = nbest;
    c.digest[t] = d;
}

// python/leaf_values.py:631-689 for one hero hand: the tuples in order,
// 1 per win and 1/k per k-way tie over the tuples without a shared card
SSB_HD void ratio_at(long i, const Ctx &c) {
    const unsigned hs = c.strength[i];
    double out = -1.0;
    if (hs != 0u) {
        const int h = static_cast<int>(i % c.mh);
        const int p = static_cast<int>((i / c.mh) % c.np);
        const long r = i / (static_cast<long>(c.mh) * c.np);
        const int *hc = c.hand_cards + (static_cast<long>(p) * c.mh + h) * 2;
        const unsigned long long hero = (1ull << hc[0]) | (1ull << hc[1]);
        const long slot = r * c.np + p;
        double wins = 0.0;
        int valid = 0;
        for (int t = c.tuple_off[slot], end = c.tuple_off[slot + 1]; t < end; ++t) {
            const Digest d = c.digest[t];
            if (d.mask & hero) continue;
            ++valid;
            if (hs > d.best)
                wins = dadd(wins, 1.0);
            else if (hs == d.best)
                wins = dadd(wins, ddiv(1.0, static_cast<double>(1u + d.nbest)));
        }
        if (valid > 0) out = ddiv(wins, static_cast<double>(valid));
    }
    c.ratio[i] = out;
}

// python/leaf_values.py:768-790: sum over the runouts in order, then divide by their count
SSB_HD void equity_at(long i, const Ctx &c) {
    const int h = static_cast<int>(i % c.mh);
    const int p = static_cast<int>(i / c.mh);
    double raw = 0.0, cnt = 0.0;
    for (int r = 0; r < c.nr; ++r) {
        const double v = c.ratio[(static_cast<long>(r) * c.np + p) * c.mh + h];
        if (v >= 0.0) {
            raw = dadd(raw, v);
            cnt = dadd(cnt, 1.0);
        }
    }
    c.equity[i] = cnt > 0.0 ? ddiv(raw, cnt) : raw;
}

// python/leaf_values.py:795-814: element i of the rows starting at row0
SSB_HD void value_at(long i, long row0, const Ctx &c) {
    const long per_row = static_cast<long>(c.np) * c.mh;
    const long row = row0 + i / per_row;
    const int p = static_cast<int>((i % per_row) / c.mh);
    const int h = static_cast<int>(i % c.mh);
    const long leaf = row / c.per;
    const int combo = static_cast<int>(row % c.per);
    float v = 0.0f;
    if (c.row_set[leaf] && h < c.nh[p]) {
        const double x = biased_value(c.equity[static_cast<long>(p) * c.mh + h], c.row_pot[leaf],
                                      (combo >> (2 * p)) & 3, opponent_profile(combo, p, c.np));
#if defined(__CUDA_ARCH__)
        v = __double2float_rn(x);
#else
        v = static_cast<float>(x);
#endif
    }
    c.values[i] = v;
}

}  // namespace leaf
}  // namespace ssb
