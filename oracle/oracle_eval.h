/*
 * oracle_eval.h -- CPU restatement of the reference 7-card hand evaluator.
 *
 * TEST INFRASTRUCTURE ONLY.  This file belongs to the oracle: only the test
 * suite, the smoke check and the CPU-baseline leg of bench.py may use it, and
 * only as a checker.  The product path never links it.
 *
 * Card encoding: card = rank*4 + suit, rank 0..12 = 2..A, suit 0..3 = c,d,h,s
 * (reference src/hand_eval.h:17-24).
 *
 * Strength encoding: category << 20 | kicker nibbles, higher is better, with
 * categories 1 = high card .. 9 = straight flush (reference src/hand_eval.h:26-35).
 * orc_eval5 follows src/hand_eval.h:40-131 step by step (sort ranks descending,
 * flush / straight / wheel tests, rank-count scan from the top); orc_eval7 is
 * the maximum over the 21 five-card subsets (src/hand_eval.h:138-156).  The
 * device copy in the reference solver (src/cuda/street_solve.cu:467-510) is the
 * same function.
 */
#ifndef ORACLE_EVAL_H
#define ORACLE_EVAL_H

#include <stdint.h>

static inline uint32_t orc_eval5(int c0, int c1, int c2, int c3, int c4)
{
    int r[5] = {c0 >> 2, c1 >> 2, c2 >> 2, c3 >> 2, c4 >> 2};
    int s[5] = {c0 & 3, c1 & 3, c2 & 3, c3 & 3, c4 & 3};
    /* descending insertion sort of the five ranks */
    for (int i = 1; i < 5; i++) {
        int v = r[i], j = i - 1;
        while (j >= 0 && r[j] < v) { r[j + 1] = r[j]; j--; }
        r[j + 1] = v;
    }
    int flush = s[0] == s[1] && s[1] == s[2] && s[2] == s[3] && s[3] == s[4];
    int straight = 0, high = r[0];
    if (r[0] - r[4] == 4 && r[0] != r[1] && r[1] != r[2] && r[2] != r[3] && r[3] != r[4])
        straight = 1;
    if (r[0] == 12 && r[1] == 3 && r[2] == 2 && r[3] == 1 && r[4] == 0) {
        straight = 1;
        high = 3; /* five-high wheel */
    }
    if (straight && flush) return (9u << 20) | ((uint32_t)high << 16);
    if (flush)
        return (6u << 20) | ((uint32_t)r[0] << 16) | ((uint32_t)r[1] << 12) |
               ((uint32_t)r[2] << 8) | ((uint32_t)r[3] << 4) | (uint32_t)r[4];
    if (straight) return (5u << 20) | ((uint32_t)high << 16);

    int cnt[13] = {0};
    for (int i = 0; i < 5; i++) cnt[r[i]]++;
    int quad = -1, trip = -1, pa = -1, pb = -1;
    for (int k = 12; k >= 0; k--) {
        if (cnt[k] == 4) quad = k;
        else if (cnt[k] == 3) trip = k;
        else if (cnt[k] == 2) { if (pa < 0) pa = k; else pb = k; }
    }
    if (quad >= 0) {
        int kick = -1;
        for (int k = 12; k >= 0; k--) if (cnt[k] > 0 && k != quad) { kick = k; break; }
        return (8u << 20) | ((uint32_t)quad << 16) | ((uint32_t)kick << 12);
    }
    if (trip >= 0 && pa >= 0) return (7u << 20) | ((uint32_t)trip << 16) | ((uint32_t)pa << 12);
    if (trip >= 0) {
        int k0 = -1, k1 = -1;
        for (int k = 12; k >= 0; k--)
            if (cnt[k] > 0 && k != trip) { if (k0 < 0) k0 = k; else k1 = k; }
        return (4u << 20) | ((uint32_t)trip << 16) | ((uint32_t)k0 << 12) | ((uint32_t)k1 << 8);
    }
    if (pa >= 0 && pb >= 0) {
        int kick = -1;
        for (int k = 12; k >= 0; k--)
            if (cnt[k] > 0 && k != pa && k != pb) { kick = k; break; }
        return (3u << 20) | ((uint32_t)pa << 16) | ((uint32_t)pb << 12) | ((uint32_t)kick << 8);
    }
    if (pa >= 0) {
        int kk[3], n = 0;
        for (int k = 12; k >= 0 && n < 3; k--) if (cnt[k] > 0 && k != pa) kk[n++] = k;
        return (2u << 20) | ((uint32_t)pa << 16) | ((uint32_t)kk[0] << 12) |
               ((uint32_t)kk[1] << 8) | ((uint32_t)kk[2] << 4);
    }
    return (1u << 20) | ((uint32_t)r[0] << 16) | ((uint32_t)r[1] << 12) |
           ((uint32_t)r[2] << 8) | ((uint32_t)r[3] << 4) | (uint32_t)r[4];
}

static inline uint32_t orc_eval7(const int c[7])
{
    uint32_t best = 0;
    /* every 5-subset of 7 = leave out an unordered pair (i, j) */
    for (int i = 0; i < 7; i++)
        for (int j = i + 1; j < 7; j++) {
            int k[5], n = 0;
            for (int m = 0; m < 7; m++) if (m != i && m != j) k[n++] = c[m];
            uint32_t v = orc_eval5(k[0], k[1], k[2], k[3], k[4]);
            if (v > best) best = v;
        }
    return best;
}

#endif
