/*
 * ss_oracle.c -- CPU oracle for the single-street N-player Linear-CFR solver.
 *
 * TEST INFRASTRUCTURE ONLY (see ss_oracle.h).  Restates the reference path
 * src/cuda/street_solve.cu on the host:
 *   - betting-tree construction      street_solve.cu:42-331
 *   - continuation-leaf expansion    street_solve.cu:336-460
 *   - BFS levels and classification  street_solve.cu:1238-1287
 *   - hand strengths                 street_solve.cu:513-550 (eval: src/hand_eval.h)
 *   - CFR kernels and host loop      street_solve.cu:575-1185, 1471-1550
 *   - output extraction              street_solve.cu:1556-1612
 * The CFR part lives in ss_oracle_impl.h, compiled once in float (the
 * reference arithmetic, same operation order) and once in double.
 */
#include "ss_oracle.h"
#include "oracle_eval.h"

#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ */
/* Tree construction                                                    */
/* ------------------------------------------------------------------ */

typedef struct {
    OrcNode *nodes;
    int n, cap;
    int *kids;
    int nk, kcap;
    int leaves;
    /* fixed inputs of one build */
    int is_river, np, max_raises;
    const int *order;
    const float *sizes;
    int nsizes;
    const int *board;
    int nboard;
} Builder;

static int b_node(Builder *b)
{
    if (b->n == b->cap) {
        b->cap = b->cap ? 2 * b->cap : 512;
        b->nodes = (OrcNode *)realloc(b->nodes, (size_t)b->cap * sizeof(OrcNode));
    }
    OrcNode *x = &b->nodes[b->n];
    memset(x, 0, sizeof(*x));
    x->player = -1;
    x->leaf_idx = -1;
    x->fold_player = -1;
    return b->n++;
}

static int b_kids(Builder *b, int count)
{
    while (b->nk + count > b->kcap) {
        b->kcap = b->kcap ? 2 * b->kcap : 2048;
        b->kids = (int *)realloc(b->kids, (size_t)b->kcap * sizeof(int));
    }
    int at = b->nk;
    b->nk += count;
    return at;
}

/* pot, bets (first np entries), board and active flags of a node
 * (street_solve.cu:85-96, 161-164) */
static void b_fill(Builder *b, int idx, int pot, const int *bets, const int *active)
{
    OrcNode *x = &b->nodes[idx];
    x->pot = pot;
    for (int i = 0; i < b->np; i++) x->bets[i] = bets[i];
    for (int i = 0; i < b->nboard && i < 5; i++) x->board_cards[i] = b->board[i];
    x->num_board = b->nboard;
    x->num_players = 0;
    for (int i = 0; i < b->np && i < ORC_MAX_PLAYERS; i++) {
        x->active_players[i] = active[i];
        if (active[i]) x->num_players++;
    }
}

/* next seat in acting order (cyclic) whose player is still in the hand
 * (street_solve.cu:106-115) */
static int next_seat(const Builder *b, const int *active, int seat)
{
    for (int i = 1; i <= b->np; i++) {
        int s = (seat + i) % b->np;
        int p = b->order[s];
        if (p < b->np && active[p]) return s;
    }
    return -1;
}

static int highest_bet(const Builder *b, const int *bets, const int *active)
{
    int m = 0;
    for (int i = 0; i < b->np; i++)
        if (active[i] && bets[i] > m) m = bets[i];
    return m;
}

/* recursive betting tree, street_solve.cu:144-331 */
static int b_build(Builder *b, int seat, int pot, int stack, const int *bets,
                   const int *acted, const int *active, int raises)
{
    int live = 0;
    for (int i = 0; i < b->np; i++) live += active[i] ? 1 : 0;

    if (live <= 1) { /* everyone else folded: fold terminal won by the survivor */
        int idx = b_node(b);
        b->nodes[idx].type = ORC_NODE_FOLD;
        for (int i = 0; i < b->np; i++)
            if (active[i]) { b->nodes[idx].player = i; break; }
        b_fill(b, idx, pot, bets, active);
        return idx;
    }

    int top = highest_bet(b, bets, active);
    int done = 1;
    for (int i = 0; i < b->np; i++) {
        if (!active[i]) continue;
        if (!acted[i] || bets[i] != top) { done = 0; break; }
    }
    if (done) { /* betting round over: showdown on the river, else a leaf */
        int idx = b_node(b);
        if (b->is_river) {
            b->nodes[idx].type = ORC_NODE_SHOWDOWN;
        } else {
            b->nodes[idx].type = ORC_NODE_LEAF;
            b->nodes[idx].leaf_idx = b->leaves++;
        }
        b_fill(b, idx, pot, bets, active);
        return idx;
    }

    int actor = b->order[seat];
    if (!active[actor]) {
        int s = next_seat(b, active, seat);
        if (s < 0) {
            int idx = b_node(b);
            b->nodes[idx].type = ORC_NODE_SHOWDOWN;
            b_fill(b, idx, pot, bets, active);
            return idx;
        }
        return b_build(b, s, pot, stack, bets, acted, active, raises);
    }

    int me = b_node(b);
    b->nodes[me].type = ORC_NODE_DECISION;
    b->nodes[me].player = actor;
    b_fill(b, me, pot, bets, active);

    int to_call = top - bets[actor];
    if (to_call < 0) to_call = 0;
    int kids[16];
    int nk = 0;
    int nxt = next_seat(b, active, seat);
    if (nxt < 0) nxt = seat;

    if (to_call > 0) { /* fold */
        int act2[ORC_MAX_PLAYERS];
        memcpy(act2, active, sizeof(act2));
        act2[actor] = 0;
        kids[nk++] = b_build(b, nxt, pot, stack, bets, acted, act2, raises);
    }
    { /* check / call */
        int bet2[ORC_MAX_PLAYERS], acted2[ORC_MAX_PLAYERS];
        memcpy(bet2, bets, sizeof(bet2));
        memcpy(acted2, acted, sizeof(acted2));
        bet2[actor] = top;
        acted2[actor] = 1;
        kids[nk++] = b_build(b, nxt, pot + to_call, stack, bet2, acted2, active, raises);
    }
    if (raises < b->max_raises && nk < 14) {
        int allin_seen = 0;
        for (int i = 0; i < b->nsizes && nk < 14; i++) {
            int amount;
            if (to_call == 0)
                amount = (int)(b->sizes[i] * (float)pot);
            else
                amount = to_call + (int)(b->sizes[i] * (float)(pot + to_call));
            if (amount >= stack) amount = stack;
            if (amount <= to_call) continue;
            if (amount >= stack) {
                if (allin_seen) continue;
                allin_seen = 1;
            }
            int bet2[ORC_MAX_PLAYERS], acted2[ORC_MAX_PLAYERS];
            memcpy(bet2, bets, sizeof(bet2));
            memcpy(acted2, acted, sizeof(acted2));
            bet2[actor] = top + amount;
            acted2[actor] = 1;
            for (int p = 0; p < b->np; p++)
                if (p != actor && active[p]) acted2[p] = 0;
            kids[nk++] = b_build(b, nxt, pot + amount, stack, bet2, acted2, active, raises + 1);
        }
        if (!allin_seen && stack > to_call && nk < 14) { /* explicit all-in */
            int bet2[ORC_MAX_PLAYERS], acted2[ORC_MAX_PLAYERS];
            memcpy(bet2, bets, sizeof(bet2));
            memcpy(acted2, acted, sizeof(acted2));
            bet2[actor] = top + stack;
            acted2[actor] = 1;
            for (int p = 0; p < b->np; p++)
                if (p != actor && active[p]) acted2[p] = 0;
            kids[nk++] = b_build(b, nxt, pot + stack, stack, bet2, acted2, active, raises + 1);
        }
    }
    int at = b_kids(b, nk);
    for (int i = 0; i < nk; i++) b->kids[at + i] = kids[i];
    b->nodes[me].first_child = at;
    b->nodes[me].num_children = nk;
    return me;
}

/* continuation expansion, street_solve.cu:336-460: every leaf becomes a chain
 * of decisions, one per active player in seat-index order, 4 children each;
 * the 4^n bottom nodes are the new leaves, numbered in creation order. */
static void b_expand(Builder *b)
{
    int orig = b->n;
    int *leaf_ids = (int *)malloc((size_t)(orig > 0 ? orig : 1) * sizeof(int));
    int nl = 0;
    for (int i = 0; i < orig; i++)
        if (b->nodes[i].type == ORC_NODE_LEAF) leaf_ids[nl++] = i;
    b->leaves = 0;

    for (int li = 0; li < nl; li++) {
        OrcNode src = b->nodes[leaf_ids[li]]; /* copy: the array may move */
        int who[ORC_MAX_PLAYERS], nw = 0;
        for (int p = 0; p < b->np; p++)
            if (src.active_players[p]) who[nw++] = p;
        if (nw == 0) continue;

        b->nodes[leaf_ids[li]].type = ORC_NODE_DECISION;
        b->nodes[leaf_ids[li]].player = who[0];
        b->nodes[leaf_ids[li]].leaf_idx = -1;

        int *par = (int *)malloc(sizeof(int));
        par[0] = leaf_ids[li];
        int npar = 1;
        for (int lev = 0; lev < nw; lev++) {
            int last = (lev == nw - 1);
            int *nxt = (int *)malloc((size_t)npar * 4 * sizeof(int));
            int nn = 0;
            for (int pi = 0; pi < npar; pi++) {
                int parent = par[pi];
                if (lev > 0) {
                    b->nodes[parent].type = ORC_NODE_DECISION;
                    b->nodes[parent].player = who[lev];
                }
                int ch[4];
                for (int s = 0; s < 4; s++) {
                    int x = b_node(b);
                    OrcNode *nx = &b->nodes[x];
                    if (last) {
                        nx->type = ORC_NODE_LEAF;
                        nx->leaf_idx = b->leaves++;
                    }
                    nx->pot = src.pot;
                    memcpy(nx->bets, src.bets, sizeof(nx->bets));
                    for (int i = 0; i < src.num_board && i < 5; i++)
                        nx->board_cards[i] = src.board_cards[i];
                    nx->num_board = src.num_board;
                    nx->num_players = 0;
                    for (int i = 0; i < b->np && i < ORC_MAX_PLAYERS; i++) {
                        nx->active_players[i] = src.active_players[i];
                        if (src.active_players[i]) nx->num_players++;
                    }
                    ch[s] = x;
                    if (!last) nxt[nn++] = x;
                }
                int at = b_kids(b, 4);
                for (int s = 0; s < 4; s++) b->kids[at + s] = ch[s];
                b->nodes[parent].first_child = at;
                b->nodes[parent].num_children = 4;
            }
            free(par);
            par = nxt;
            npar = nn;
        }
        free(par);
    }
    free(leaf_ids);
}

int orc_build_tree(const int *board, int num_board, int starting_pot, int effective_stack,
                   const float *bet_sizes, int num_bet_sizes, int num_players,
                   const int *acting_order, int is_river, int use_cont_strats,
                   int max_raises, OrcTree *out)
{
    memset(out, 0, sizeof(*out));
    if (num_players < 1 || num_players > ORC_MAX_PLAYERS) return -1;
    Builder b;
    memset(&b, 0, sizeof(b));
    b.is_river = is_river;
    b.np = num_players;
    b.max_raises = max_raises;
    b.order = acting_order;
    b.sizes = bet_sizes;
    b.nsizes = num_bet_sizes;
    b.board = board;
    b.nboard = num_board;

    int bets[ORC_MAX_PLAYERS] = {0}, acted[ORC_MAX_PLAYERS] = {0}, active[ORC_MAX_PLAYERS] = {0};
    for (int i = 0; i < num_players; i++) active[i] = 1;
    b_build(&b, 0, starting_pot, effective_stack, bets, acted, active, 0);
    if (use_cont_strats && !is_river && b.leaves > 0) b_expand(&b);

    out->nodes = b.nodes;
    out->children = b.kids;
    out->num_nodes = b.n;
    out->num_children_total = b.nk;
    out->num_leaves = b.leaves;
    out->num_players = num_players;
    out->is_river = is_river;
    out->starting_pot = starting_pot;
    out->effective_stack = effective_stack;
    for (int i = 0; i < num_board && i < 5; i++) out->board[i] = board[i];
    out->num_board = num_board;

    /* BFS order and depths from node 0 (street_solve.cu:1238-1259) */
    int n = b.n;
    out->level_order = (int *)malloc((size_t)n * sizeof(int));
    out->node_depth = (int *)calloc((size_t)n, sizeof(int));
    int head = 0, tail = 0;
    out->level_order[tail++] = 0;
    while (head < tail) {
        int x = out->level_order[head++];
        int d = out->node_depth[x];
        if (d > out->max_depth) out->max_depth = d;
        for (int a = 0; a < b.nodes[x].num_children; a++) {
            int c = b.kids[b.nodes[x].first_child + a];
            out->node_depth[c] = d + 1;
            out->level_order[tail++] = c;
        }
    }
    return 0;
}

void orc_free_tree(OrcTree *t)
{
    free(t->nodes);
    free(t->children);
    free(t->level_order);
    free(t->node_depth);
    memset(t, 0, sizeof(*t));
}

uint32_t orc_eval7_cards(const int *cards7) { return orc_eval7(cards7); }

/* ------------------------------------------------------------------ */
/* CFR in float (reference arithmetic) and in double                   */
/* ------------------------------------------------------------------ */

#define REAL float
#define RSUF(name) name##_f32
#define RLIT(x) x##f
#include "ss_oracle_impl.h"
#undef REAL
#undef RSUF
#undef RLIT

#define REAL double
#define RSUF(name) name##_f64
#define RLIT(x) x
#include "ss_oracle_impl.h"
#undef REAL
#undef RSUF
#undef RLIT

int orc_solve_f64_closed(const OrcTree *t, const int *hands, const float *weights,
                         const int *num_hands, const float *leaf_values, const int *frozen,
                         int iterations, double *root_strategy, double *root_ev,
                         double *avg_strategies, int *avg_node_ids, double *regrets_out,
                         double *strategy_sum_out)
{
    return solve_impl_f64(t, hands, weights, num_hands, leaf_values, frozen, iterations,
                          root_strategy, root_ev, avg_strategies, avg_node_ids, regrets_out,
                          strategy_sum_out, 1);
}

/* ------------------------------------------------------------------ */
/* FP64 best response and exploitability                               */
/* ------------------------------------------------------------------ */

/* Counterfactual values for one traverser under a fixed profile, FP64.
 * The profile's reach and the terminal values follow the reference kernels
 * (same opponent sets, card-removal rules and payoffs); at the traverser's
 * own nodes the value is the profile-weighted sum (mode 0) or the best
 * action (mode 1, a pure best response per information set). */
static void orc_profile_pass(OrcCtx_f64 *c, const float *weights, const float *leaf_values,
                             const int *frozen, int trav, int mode)
{
    const OrcTree *t = c->t;
    for (int rp = 0; rp < c->np; rp++) {
        if (rp == trav) continue;
        double *r = &c->reach[(size_t)rp * c->N * c->max_h];
        memset(r, 0, (size_t)c->N * c->max_h * sizeof(double));
        for (int h = 0; h < c->nh[rp]; h++) r[h] = (double)weights[(size_t)rp * c->max_h + h];
        for (int i = 0; i < c->N; i++) prop_reach_f64(c, t->level_order[i], rp);
    }
    terminals_f64(c, trav, leaf_values);
    for (int i = c->N - 1; i >= 0; i--) {
        int n = t->level_order[i];
        const OrcNode *x = &t->nodes[n];
        if (x->type != ORC_NODE_DECISION) continue;
        int na = x->num_children;
        for (int h = 0; h < c->nh[trav]; h++) {
            double v = 0;
            if (x->player == trav && mode == 1) {
                int fa = frozen ? frozen[n] : -1;
                if (fa >= 0 && fa < na) {
                    v = c->cfv[(size_t)t->children[x->first_child + fa] * c->max_h + h];
                } else {
                    v = -1e300;
                    for (int a = 0; a < na; a++) {
                        double cv = c->cfv[(size_t)t->children[x->first_child + a] * c->max_h + h];
                        if (cv > v) v = cv;
                    }
                }
            } else if (x->player == trav) {
                for (int a = 0; a < na; a++)
                    v += c->strategy[((size_t)n * ORC_MAX_ACTIONS + a) * c->max_h + h] *
                         c->cfv[(size_t)t->children[x->first_child + a] * c->max_h + h];
            } else {
                for (int a = 0; a < na; a++)
                    v += c->cfv[(size_t)t->children[x->first_child + a] * c->max_h + h];
            }
            c->cfv[(size_t)n * c->max_h + h] = v;
        }
    }
}

static void orc_load_profile(OrcCtx_f64 *c, const float *avg, const int *frozen)
{
    const OrcTree *t = c->t;
    int di = 0;
    for (int i = 0; i < c->N; i++) {
        const OrcNode *x = &t->nodes[i];
        if (x->type != ORC_NODE_DECISION) continue;
        for (int a = 0; a < ORC_MAX_ACTIONS; a++)
            for (int h = 0; h < c->max_h; h++)
                c->strategy[((size_t)i * ORC_MAX_ACTIONS + a) * c->max_h + h] =
                    (double)avg[((size_t)di * ORC_MAX_ACTIONS + a) * c->max_h + h];
        if (frozen) freeze_f64(c, frozen, i);
        di++;
    }
}

int orc_profile_cfv(const OrcTree *t, const int *hands, const float *weights,
                    const int *num_hands, const float *leaf_values, const int *frozen,
                    const float *avg_strategies, int traverser, int mode, double *cfv_root)
{
    OrcCtx_f64 c;
    int *sd = NULL, nsd = 0;
    if (ctx_init_f64(&c, t, hands, num_hands, &sd, &nsd) != 0) return -1;
    orc_load_profile(&c, avg_strategies, frozen);
    orc_profile_pass(&c, weights, leaf_values, frozen, traverser, mode);
    for (int h = 0; h < c.max_h; h++) cfv_root[h] = c.cfv[h];
    free(sd);
    ctx_free_f64(&c);
    return 0;
}

double orc_exploitability(const OrcTree *t, const int *hands, const float *weights,
                          const int *num_hands, const float *leaf_values, const int *frozen,
                          const float *avg_strategies, double *br_value, double *cur_value,
                          double *deal_mass)
{
    OrcCtx_f64 c;
    int *sd = NULL, nsd = 0;
    if (ctx_init_f64(&c, t, hands, num_hands, &sd, &nsd) != 0) return -1.0;
    orc_load_profile(&c, avg_strategies, frozen);
    int np = c.np, H = c.max_h;
    double nash = 0;
    for (int p = 0; p < np; p++) {
        double vals[2];
        for (int mode = 0; mode < 2; mode++) {
            orc_profile_pass(&c, weights, leaf_values, frozen, p, mode);
            double u = 0;
            for (int h = 0; h < num_hands[p]; h++)
                u += (double)weights[(size_t)p * H + h] * c.cfv[h];
            vals[mode] = u;
        }
        if (cur_value) cur_value[p] = vals[0];
        if (br_value) br_value[p] = vals[1];
        nash += vals[1] - vals[0];
    }
    /* valid-deal mass: sum over pairwise card-disjoint, board-free hand tuples
     * (one hand per player) of the product of the range weights */
    double z = 0;
    int idx[ORC_MAX_PLAYERS] = {0};
    const OrcNode *root = &t->nodes[0];
    for (;;) {
        int used[ORC_MAX_PLAYERS][2];
        double prod = 1.0;
        int ok = 1;
        for (int p = 0; p < np && ok; p++) {
            int a0 = hands[((size_t)p * H + idx[p]) * 2], a1 = hands[((size_t)p * H + idx[p]) * 2 + 1];
            used[p][0] = a0;
            used[p][1] = a1;
            if (board_blocked_f64(root, a0, a1)) { ok = 0; break; }
            for (int q = 0; q < p; q++)
                if (a0 == used[q][0] || a0 == used[q][1] || a1 == used[q][0] || a1 == used[q][1]) {
                    ok = 0;
                    break;
                }
            prod *= (double)weights[(size_t)p * H + idx[p]];
        }
        if (ok) z += prod;
        int k = np - 1;
        while (k >= 0) {
            if (++idx[k] < num_hands[k]) break;
            idx[k] = 0;
            k--;
        }
        if (k < 0) break;
    }
    if (deal_mass) *deal_mass = z;
    free(sd);
    ctx_free_f64(&c);
    return z > 0 ? nash / z : 0.0;
}

/* ------------------------------------------------------------------ */
/* all-hands checksum of the evaluator restatement                     */
/* ------------------------------------------------------------------ */

static uint64_t orc_mix64(uint64_t z)
{
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

/* sum (mod 2^64) over every 7-card set of mix64(card mask) * orc_eval7, and
 * the per-category counts */
uint64_t orc_eval7_checksum(uint64_t *hist)
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
                uint32_t s = orc_eval7(c);
                uint64_t m = 0;
                for (int k = 0; k < 7; k++) m |= 1ull << c[k];
                local += orc_mix64(m) * (uint64_t)s;
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

void orc_eval7_many(const int *cards, long n, uint32_t *out)
{
    for (long i = 0; i < n; i++) out[i] = orc_eval7(cards + 7 * i);
}
