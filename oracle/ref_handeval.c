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
