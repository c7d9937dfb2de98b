// ss_rank.cuh -- integer 7-card hand ranker.
//
// Produces exactly the reference strength encoding (src/hand_eval.h:26-35):
// category << 20 | rank nibbles, higher is better, categories 1 = high card
// .. 9 = straight flush, where the reference takes the maximum of its 5-card
// evaluator over the 21 subsets (src/hand_eval.h:138-156).  Instead of 21
// sorts, this ranker works on 13-bit rank masks: one mask per suit, one for
// all ranks, and per-rank counts.  With seven cards a flush excludes quads
// and full houses (either would need a sixth card of the flush suit), so the
// categories are tested in descending order on those masks.
#pragma once

#include <cstdint>

#if defined(__CUDACC__)
#define SSB_HD __host__ __device__ __forceinline__
#else
#define SSB_HD inline
#endif

namespace ssb {

// highest rank r such that ranks r-4..r are all in mask; the five-high wheel
// (A,2,3,4,5) gives 3; -1 if no straight
SSB_HD int straight_top(unsigned mask) {
    for (int r = 12; r >= 4; --r)
        if (((mask >> (r - 4)) & 0x1Fu) == 0x1Fu) return r;
    if ((mask & 0x100Fu) == 0x100Fu) return 3;
    return -1;
}

// the n highest ranks present in mask (n <= 5), packed as nibbles from bit 16 down
SSB_HD uint32_t top_ranks(unsigned mask, int n) {
    uint32_t v = 0;
    int shift = 16;
    for (int r = 12; r >= 0 && n > 0; --r)
        if (mask & (1u << r)) {
            v |= static_cast<uint32_t>(r) << shift;
            shift -= 4;
            --n;
        }
    return v;
}

// cards: 0..51, card = rank * 4 + suit; the seven cards must be distinct
SSB_HD uint32_t rank7(const int c[7]) {
    unsigned suit_mask[4] = {0u, 0u, 0u, 0u};
    int count[13];
    for (int r = 0; r < 13; ++r) count[r] = 0;
    for (int i = 0; i < 7; ++i) {
        suit_mask[c[i] & 3] |= 1u << (c[i] >> 2);
        count[c[i] >> 2]++;
    }
    for (int s = 0; s < 4; ++s) {
        unsigned m = suit_mask[s];
        int n = 0;
        for (int r = 0; r < 13; ++r) n += (m >> r) & 1u;
        if (n >= 5) {
            int sf = straight_top(m);
            if (sf >= 0) return (9u << 20) | (static_cast<uint32_t>(sf) << 16);
            return (6u << 20) | top_ranks(m, 5);
        }
    }
    unsigned all = suit_mask[0] | suit_mask[1] | suit_mask[2] | suit_mask[3];
    // quads; the highest trip rank and a second one (which can only play as a pair);
    // ranks holding exactly two cards in descending order
    int quad = -1, trip = -1, trip2 = -1;
    int pairs[3], np = 0;
    for (int r = 12; r >= 0; --r) {
        if (count[r] == 4 && quad < 0) quad = r;
        if (count[r] == 3) {
            if (trip < 0) trip = r;
            else if (trip2 < 0) trip2 = r;
        }
        if (count[r] == 2 && np < 3) pairs[np++] = r;
    }
    if (quad >= 0) {
        unsigned rest = all & ~(1u << quad);
        return (8u << 20) | (static_cast<uint32_t>(quad) << 16) | (top_ranks(rest, 1) >> 4);
    }
    if (trip >= 0) {
        // full house: best pair among a second trip rank and the real pairs
        int fh_pair = trip2;
        if (np > 0 && pairs[0] > fh_pair) fh_pair = pairs[0];
        if (fh_pair >= 0)
            return (7u << 20) | (static_cast<uint32_t>(trip) << 16) |
                   (static_cast<uint32_t>(fh_pair) << 12);
    }
    int st = straight_top(all);
    if (st >= 0) return (5u << 20) | (static_cast<uint32_t>(st) << 16);
    if (trip >= 0) {
        unsigned rest = all & ~(1u << trip);
        return (4u << 20) | (static_cast<uint32_t>(trip) << 16) | (top_ranks(rest, 2) >> 4);
    }
    if (np >= 2) {
        unsigned rest = all & ~(1u << pairs[0]) & ~(1u << pairs[1]);
        return (3u << 20) | (static_cast<uint32_t>(pairs[0]) << 16) |
               (static_cast<uint32_t>(pairs[1]) << 12) | (top_ranks(rest, 1) >> 8);
    }
    if (np == 1) {
        unsigned rest = all & ~(1u << pairs[0]);
        return (2u << 20) | (static_cast<uint32_t>(pairs[0]) << 16) | (top_ranks(rest, 3) >> 4);
    }
    return (1u << 20) | top_ranks(all, 5);
}

}  // namespace ssb
