// ss_leaf_plan.cpp -- host plan of the continuation-value producer (see
// ss_leaf.h).  No CUDA here: the plan fixes the runouts' board cards, the
// live hands, the opponent tuples each hero player is scored against and
// the output rows, exactly as the reference's Python loops choose them.
#include "ss_leaf.h"

#include <cmath>
#include <new>

namespace ssb {
namespace leaf {

// ---------------------------------------------------------------------------
// MT19937 (Matsumoto & Nishimura, 1998) with init_by_array seeding
// ---------------------------------------------------------------------------

PyRandom::PyRandom(uint32_t seed) {
    // init_genrand(19650218)
    mt_[0] = 19650218u;
    for (int k = 1; k < kN; ++k) mt_[k] = 1812433253u * (mt_[k - 1] ^ (mt_[k - 1] >> 30)) + static_cast<uint32_t>(k);
    // init_by_array with the key {seed}
    int i = 1;
    for (int k = kN; k > 0; --k) {
        mt_[i] = (mt_[i] ^ ((mt_[i - 1] ^ (mt_[i - 1] >> 30)) * 1664525u)) + seed;   // key[0] + j, j = 0
        if (++i >= kN) {
            mt_[0] = mt_[kN - 1];
            i = 1;
        }
    }
    for (int k = kN - 1; k > 0; --k) {
        mt_[i] = (mt_[i] ^ ((mt_[i - 1] ^ (mt_[i - 1] >> 30)) * 1566083941u)) - static_cast<uint32_t>(i);
        if (++i >= kN) {
            mt_[0] = mt_[kN - 1];
            i = 1;
        }
    }
    mt_[0] = 0x80000000u;
    i_ = kN;
}

uint32_t PyRandom::next32() {
    constexpr int kM = 397;
    constexpr uint32_t kMatrix = 0x9908b0dfu, kUpper = 0x80000000u, kLower = 0x7fffffffu;
    if (i_ >= kN) {
        for (int k = 0; k < kN; ++k) {
            const uint32_t y = (mt_[k] & kUpper) | (mt_[(k + 1) % kN] & kLower);
            mt_[k] = mt_[(k + kM) % kN] ^ (y >> 1) ^ ((y & 1u) ? kMatrix : 0u);
        }
        i_ = 0;
    }
    uint32_t y = mt_[i_++];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
}

uint32_t PyRandom::below(uint32_t n) {
    int k = 0;
    while (k < 32 && (n >> k) != 0u) ++k;   // n.bit_length()
    const int shift = 32 - k;
    uint32_t r = next32() >> shift;
    while (r >= n) r = next32() >> shift;
    return r;
}

int opponent_tuples(int nopp, const int *sizes, std::vector<int> *out) {
    long long total = 1;
    for (int k = 0; k < nopp; ++k) {
        if (sizes[k] <= 0) return 0;
        total *= sizes[k];   // <= 1326^5, no overflow
    }
    if (total <= kTupleLimit) {
        std::vector<int> pos(static_cast<size_t>(nopp), 0);
        for (long long t = 0; t < total; ++t) {
            out->insert(out->end(), pos.begin(), pos.end());
            for (int k = nopp - 1; k >= 0; --k) {   // odometer, last opponent fastest
                if (++pos[static_cast<size_t>(k)] < sizes[k]) break;
                pos[static_cast<size_t>(k)] = 0;
            }
        }
        return static_cast<int>(total);
    }
    PyRandom rng(42u);
    for (int t = 0; t < kTupleLimit; ++t)
        for (int k = 0; k < nopp; ++k) out->push_back(static_cast<int>(rng.below(static_cast<uint32_t>(sizes[k]))));
    return kTupleLimit;
}

// ---------------------------------------------------------------------------
// plan
// ---------------------------------------------------------------------------

namespace {
bool valid_card(int c) { return c >= 0 && c < 52; }
}  // namespace

int make_plan(const SSLeafValueInput *in, Plan *plan, std::string *err) {
    auto bad = [err](const std::string &m) {
        *err = "ss_leaf_values_gpu: " + m;
        return SS_ERR_INVALID;
    };
    if (!in) return bad("null input");
    const int np = in->num_players, mh = in->max_hands;
    if (np < 2 || np > SS_MAX_PLAYERS) return bad("num_players must be 2.." + std::to_string(SS_MAX_PLAYERS));
    if (mh < 1 || mh > kMaxHands) return bad("max_hands must be 1..1326");
    if (!in->num_hands) return bad("null num_hands");
    if (in->num_board != 3 && in->num_board != 4) return bad("num_board must be 3 (flop) or 4 (turn)");
    if (!in->board) return bad("null board");
    if (in->num_runouts < 0 || (in->num_runouts > 0 && !in->runout_cards)) return bad("bad runouts");
    if (in->num_leaves < 0 || (in->num_leaves > 0 && (!in->leaf_idx || !in->leaf_pot)))
        return bad("bad leaf descriptors");
    try {
        Plan &P = *plan;
        P = Plan();
        P.np = np;
        P.mh = mh;
        P.nr = in->num_runouts;
        P.num_leaves = in->num_leaves;
        P.per = 1 << (2 * np);
        P.nh.assign(in->num_hands, in->num_hands + np);
        bool any_hands = false;
        for (int p = 0; p < np; ++p) {
            if (P.nh[p] < 0 || P.nh[p] > mh)
                return bad("num_hands[" + std::to_string(p) + "] must be 0..max_hands");
            any_hands = any_hands || P.nh[p] > 0;
        }
        if (any_hands && !in->hand_cards) return bad("null hand_cards");
        P.hand_cards.assign(static_cast<size_t>(np) * mh * 2, 0);
        for (int p = 0; p < np; ++p)
            for (int h = 0; h < P.nh[p]; ++h) {
                const size_t o = (static_cast<size_t>(p) * mh + h) * 2;
                const int a = in->hand_cards[o], b = in->hand_cards[o + 1];
                if (!valid_card(a) || !valid_card(b) || a == b)
                    return bad("hand " + std::to_string(h) + " of player " + std::to_string(p) +
                               " needs two different cards 0..51");
                P.hand_cards[o] = a;
                P.hand_cards[o + 1] = b;
            }
        const int extra = 5 - in->num_board;
        unsigned long long board_mask = 0ull;
        for (int i = 0; i < in->num_board; ++i) {
            const int c = in->board[i];
            if (!valid_card(c) || (board_mask >> c & 1ull)) return bad("board cards must be distinct, 0..51");
            board_mask |= 1ull << c;
        }
        P.board5.resize(static_cast<size_t>(P.nr) * 5);
        for (int r = 0; r < P.nr; ++r) {
            unsigned long long m = board_mask;
            for (int i = 0; i < in->num_board; ++i) P.board5[static_cast<size_t>(r) * 5 + i] = in->board[i];
            for (int i = 0; i < extra; ++i) {
                const int c = in->runout_cards[static_cast<size_t>(r) * extra + i];
                if (!valid_card(c) || (m >> c & 1ull))
                    return bad("runout " + std::to_string(r) + " repeats a card or holds one outside 0..51");
                m |= 1ull << c;
                P.board5[static_cast<size_t>(r) * 5 + in->num_board + i] = c;
            }
        }
        P.row_pot.assign(static_cast<size_t>(P.num_leaves), 0.0);
        P.row_set.assign(static_cast<size_t>(P.num_leaves), 0);
        for (int k = 0; k < in->num_leaves; ++k) {
            const int li = in->leaf_idx[k];
            if (li < 0) return bad("leaf_idx must be >= 0");
            if (!std::isfinite(in->leaf_pot[k])) return bad("leaf pots must be finite");
            if (li < P.num_leaves) {   // rows past num_leaves * 4^N are skipped, as in the reference
                P.row_pot[static_cast<size_t>(li)] = in->leaf_pot[k];
                P.row_set[static_cast<size_t>(li)] = 1;
            }
        }

        // live hands and opponent tuples per runout and hero player
        P.tuple_off.assign(static_cast<size_t>(P.nr) * np + 1, 0);
        std::vector<std::vector<int>> live(static_cast<size_t>(np));
        std::vector<int> sizes(static_cast<size_t>(np)), pos;
        for (int r = 0; r < P.nr; ++r) {
            unsigned long long m = 0ull;
            for (int i = 0; i < 5; ++i) m |= 1ull << P.board5[static_cast<size_t>(r) * 5 + i];
            for (int p = 0; p < np; ++p) {
                live[p].clear();
                for (int h = 0; h < P.nh[p]; ++h) {
                    const size_t o = (static_cast<size_t>(p) * mh + h) * 2;
                    if (!((m >> P.hand_cards[o]) & 1ull) && !((m >> P.hand_cards[o + 1]) & 1ull)) live[p].push_back(h);
                }
            }
            for (int p = 0; p < np; ++p) {
                const size_t slot = static_cast<size_t>(r) * np + p;
                int count = 0;
                if (!live[p].empty()) {
                    int k = 0;
                    for (int q = 0; q < np; ++q)
                        if (q != p) sizes[static_cast<size_t>(k++)] = static_cast<int>(live[q].size());
                    pos.clear();
                    count = opponent_tuples(np - 1, sizes.data(), &pos);
                    for (int t = 0; t < count; ++t) {
                        P.tuple_owner.push_back(static_cast<int>(slot));
                        int kk = 0;
                        for (int q = 0; q < np; ++q) {
                            if (q == p) continue;
                            const int at = pos[static_cast<size_t>(t) * (np - 1) + kk++];
                            P.tuple_hand.push_back(static_cast<uint16_t>(live[q][static_cast<size_t>(at)]));
                        }
                    }
                }
                P.tuple_off[slot + 1] = P.tuple_off[slot] + count;
            }
        }
    } catch (const std::bad_alloc &) {
        *err = "ss_leaf_values_gpu: host allocation failed";
        return SS_ERR_NOMEM;
    }
    return SS_OK;
}

}  // namespace leaf
}  // namespace ssb
