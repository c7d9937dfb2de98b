/*
 * ref_handeval.c -- exports the reference evaluator (src/hand_eval.h, found
 * through the include path at build time) from a shared library so the tests
 * can compare the oracle restatement and the device ranker against it.
 *
 * TEST INFRASTRUCTURE ONLY; built into oracle/_ref/ by oracle/build_ref.py.
 */
#include <stdint.h>
#include "hand_eval.h"

uint32_t ref_eval7(const int *cards7) { return eval7(cards7); }
uint32_t ref_eval5(int a, int b, int c, int d, int e) { return eval5(a, b, c, d, e); }

/* eval7 over many 7-card rows [n][7] */
void ref_eval7_many(const int *cards, long n, uint32_t *out)
{
    for (long i = 0; i < n; i++) out[i] = eval7(cards + 7 * i);
}

/* splitmix64 finaliser: a fixed pseudo-random weight per 52-bit card mask */
static uint64_t mix64(uint64_t z)
{
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

/* Over every 7-card set: sum (mod 2^64) of mix64(card mask) * eval7, and the
 * number of sets per category (hist[0..9]).  One order-independent number
 * that changes if any single strength changes. */
uint64_t ref_eval7_checksum(uint64_t *hist)
{
    uint64_t total = 0;
    for (int i = 0; i < 10; i++) hist[i] = 0;
#pragma omp parallel
    {
        uint64_t local = 0, lh[10] = {0};
        int c[7];
#pragma omp for schedule(dynamic)
        for (int a = 0; a < 52; a++) {
            c[0] = a;
            for (c[1] = c[0] + 1; c[1] < 52; c[1]++)
            for (c[2] = c[1] + 1; c[2] < 52; c[2]++)
            for (c[3] = c[2] + 1; c[3] < 52; c[3]++)
            for (c[4] = c[3] + 1; c[4] < 52; c[4]++)
            for (c[5] = c[4] + 1; c[5] < 52; c[5]++)
            for (c[6] = c[5] + 1; c[6] < 52; c[6]++) {
                uint32_t s = eval7(c);
                uint64_t m = 0;
                for (int k = 0; k < 7; k++) m |= 1ull << c[k];
                local += mix64(m) * (uint64_t)s;
                lh[s >> 20]++;
            }
        }
#pragma omp critical
        {
            total += local;
            for (int i = 0; i < 10; i++) hist[i] += lh[i];
        }
    }
    return total;
}
