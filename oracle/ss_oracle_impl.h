/*
 * ss_oracle_impl.h -- CFR body of the oracle, included twice by ss_oracle.c
 * with REAL = float (the reference arithmetic, same operation order as the
 * reference kernels) and REAL = double.
 *
 * TEST INFRASTRUCTURE ONLY (see ss_oracle.h).
 */

/* per-solve scratch */
typedef struct {
    const OrcTree *t;
    int np, max_h, N;
    const int *hands;     /* [np][max_h][2] */
    const int *nh;        /* [np] */
    REAL *reach;          /* [np][N][max_h] */
    REAL *cfv;            /* [N][max_h] */
    REAL *strategy;       /* [N][8][max_h] */
    uint32_t *strength;   /* [num_sd][np][max_h] */
    int *sd_local;        /* [N] */
    int closed;           /* 1: folds and leaves with 1-2 counted opponents by the
                             card-removal closed form (terminals_closed) */
} RSUF(OrcCtx);

#define OH(c, p, h, k) ((c)->hands[(((size_t)(p) * (c)->max_h + (h)) * 2) + (k)])
#define OREACH(c, p, n, h) ((c)->reach[((size_t)(p) * (c)->N + (n)) * (c)->max_h + (h)])
#define OCFV(c, n, h) ((c)->cfv[(size_t)(n) * (c)->max_h + (h)])
#define OST(arr, c, n, a, h) ((arr)[((size_t)(n) * ORC_MAX_ACTIONS + (a)) * (c)->max_h + (h)])

static int RSUF(board_blocked)(const OrcNode *x, int c0, int c1)
{
    for (int b = 0; b < x->num_board; b++)
        if (c0 == x->board_cards[b] || c1 == x->board_cards[b]) return 1;
    return 0;
}

/* regret matching at one decision node for the acting player's hands,
 * street_solve.cu:575-614.  The regret-pruning branch of the reference
 * (:594,599) replaces a regret below -1e4 by 0, which the positive part
 * below already does, so it does not change the result and is omitted. */
static void RSUF(regret_match)(RSUF(OrcCtx) *c, const REAL *regrets, int n)
{
    const OrcNode *x = &c->t->nodes[n];
    int p = x->player;
    if (x->type != ORC_NODE_DECISION || p < 0 || p >= c->np) return;
    int na = x->num_children;
    for (int h = 0; h < c->nh[p]; h++) {
        REAL sum = 0;
        for (int a = 0; a < na; a++) {
            REAL r = OST(regrets, c, n, a, h);
            sum += (r > 0) ? r : 0;
        }
        if (sum > 0) {
            REAL inv = RLIT(1.0) / sum;
            for (int a = 0; a < na; a++) {
                REAL r = OST(regrets, c, n, a, h);
                OST(c->strategy, c, n, a, h) = ((r > 0) ? r : 0) * inv;
            }
        } else {
            REAL u = RLIT(1.0) / (REAL)na;
            for (int a = 0; a < na; a++) OST(c->strategy, c, n, a, h) = u;
        }
    }
}

/* A3 freeze, street_solve.cu:621-644 */
static void RSUF(freeze)(RSUF(OrcCtx) *c, const int *frozen, int n)
{
    int fa = frozen[n];
    if (fa < 0) return;
    const OrcNode *x = &c->t->nodes[n];
    int p = x->player;
    if (p < 0 || p >= c->np) return;
    for (int h = 0; h < c->nh[p]; h++)
        for (int a = 0; a < x->num_children; a++)
            OST(c->strategy, c, n, a, h) = (a == fa) ? RLIT(1.0) : RLIT(0.0);
}

/* top-down reach of one player through one decision node,
 * street_solve.cu:650-683 */
static void RSUF(prop_reach)(RSUF(OrcCtx) *c, int n, int rp)
{
    const OrcNode *x = &c->t->nodes[n];
    if (x->type != ORC_NODE_DECISION) return;
    for (int h = 0; h < c->nh[rp]; h++) {
        REAL pr = OREACH(c, rp, n, h);
        for (int a = 0; a < x->num_children; a++) {
            int ch = c->t->children[x->first_child + a];
            OREACH(c, rp, ch, h) = (x->player == rp) ? pr * OST(c->strategy, c, n, a, h) : pr;
        }
    }
}

/* Sum over opponent-hand tuples (one hand per listed opponent) that share no
 * card with the traverser hand, the board or each other, of the product of
 * their reaches; the odometer of street_solve.cu:771-823 (fold) and
 * :1079-1127 (leaf).  With a single opponent this is the plain filtered sum of
 * :746-761 / :1047-1066. */
static REAL RSUF(opp_mass)(RSUF(OrcCtx) *c, const OrcNode *x, int node, const int *opp,
                           int n_opp, int hc0, int hc1)
{
    if (n_opp == 1) {
        int p = opp[0];
        REAL s = 0;
        for (int o = 0; o < c->nh[p]; o++) {
            int oc0 = OH(c, p, o, 0), oc1 = OH(c, p, o, 1);
            if (hc0 == oc0 || hc0 == oc1 || hc1 == oc0 || hc1 == oc1) continue;
            if (RSUF(board_blocked)(x, oc0, oc1)) continue;
            s += OREACH(c, p, node, o);
        }
        return s;
    }
    int idx[ORC_MAX_PLAYERS];
    for (int i = 0; i < n_opp; i++) idx[i] = 0;
    REAL total = 0;
    for (;;) {
        int oc[ORC_MAX_PLAYERS][2];
        REAL prod = RLIT(1.0);
        int ok = 1;
        for (int i = 0; i < n_opp && ok; i++) {
            int p = opp[i], o = idx[i];
            int a0 = OH(c, p, o, 0), a1 = OH(c, p, o, 1);
            oc[i][0] = a0;
            oc[i][1] = a1;
            if (hc0 == a0 || hc0 == a1 || hc1 == a0 || hc1 == a1) { ok = 0; break; }
            if (RSUF(board_blocked)(x, a0, a1)) { ok = 0; break; }
            prod *= OREACH(c, p, node, o);
            for (int j = 0; j < i; j++)
                if (a0 == oc[j][0] || a0 == oc[j][1] || a1 == oc[j][0] || a1 == oc[j][1]) {
                    ok = 0;
                    break;
                }
        }
        if (ok && prod > 0) total += prod;
        int k = n_opp - 1;
        while (k >= 0) {
            if (++idx[k] < c->nh[opp[k]]) break;
            idx[k] = 0;
            k--;
        }
        if (k < 0) break;
    }
    return total;
}

/* fold terminal, street_solve.cu:704-826: every non-traverser player counts,
 * folded or not */
static void RSUF(fold_value)(RSUF(OrcCtx) *c, int n, int trav)
{
    const OrcNode *x = &c->t->nodes[n];
    int opp[ORC_MAX_PLAYERS], k = 0;
    for (int p = 0; p < c->np; p++) if (p != trav) opp[k++] = p;
    REAL payoff = (trav == x->player) ? (REAL)(x->pot - x->bets[trav]) : -(REAL)x->bets[trav];
    for (int h = 0; h < c->nh[trav]; h++) {
        int hc0 = OH(c, trav, h, 0), hc1 = OH(c, trav, h, 1);
        OCFV(c, n, h) = payoff * RSUF(opp_mass)(c, x, n, opp, k, hc0, hc1);
    }
}

/* depth-limit leaf, street_solve.cu:1012-1130: active opponents only; no
 * active opponent gives mass 1 */
static void RSUF(leaf_value)(RSUF(OrcCtx) *c, int n, int trav, const float *leaf_values)
{
    const OrcNode *x = &c->t->nodes[n];
    int opp[ORC_MAX_PLAYERS], k = 0;
    for (int p = 0; p < c->np; p++) if (p != trav && x->active_players[p]) opp[k++] = p;
    for (int h = 0; h < c->nh[trav]; h++) {
        if (x->leaf_idx < 0) { OCFV(c, n, h) = 0; continue; }
        REAL ev = (REAL)leaf_values[((size_t)x->leaf_idx * c->np + trav) * c->max_h + h];
        int hc0 = OH(c, trav, h, 0), hc1 = OH(c, trav, h, 1);
        REAL m = (k == 0) ? RLIT(1.0) : RSUF(opp_mass)(c, x, n, opp, k, hc0, hc1);
        OCFV(c, n, h) = ev * m;
    }
}

/* showdown terminal, street_solve.cu:840-1005 */
static void RSUF(showdown_value)(RSUF(OrcCtx) *c, int n, int trav)
{
    const OrcNode *x = &c->t->nodes[n];
    int sd = c->sd_local[n];
    const uint32_t *str = c->strength;
#define OSTR(p, h) (str[((size_t)sd * c->np + (p)) * c->max_h + (h)])
    int opp[ORC_MAX_PLAYERS], k = 0;
    for (int p = 0; p < c->np; p++) if (p != trav && x->active_players[p]) opp[k++] = p;
    REAL pot = (REAL)x->pot;
    REAL tb = (REAL)x->bets[trav];
    for (int h = 0; h < c->nh[trav]; h++) {
        if (!x->active_players[trav]) { OCFV(c, n, h) = 0; continue; }
        uint32_t hs = OSTR(trav, h);
        if (hs == 0) { OCFV(c, n, h) = 0; continue; }
        int hc0 = OH(c, trav, h, 0), hc1 = OH(c, trav, h, 1);
        REAL val = 0;
        if (k == 1) {
            int p = opp[0];
            for (int o = 0; o < c->nh[p]; o++) {
                int oc0 = OH(c, p, o, 0), oc1 = OH(c, p, o, 1);
                if (hc0 == oc0 || hc0 == oc1 || hc1 == oc0 || hc1 == oc1) continue;
                uint32_t os = OSTR(p, o);
                if (os == 0) continue;
                REAL w = OREACH(c, p, n, o);
                if (hs > os) val += w * (pot - tb);
                else if (hs < os) val -= w * tb;
                else val += w * (pot * RLIT(0.5) - tb);
            }
            OCFV(c, n, h) = val;
            continue;
        }
        int idx[ORC_MAX_PLAYERS];
        for (int i = 0; i < k; i++) idx[i] = 0;
        for (;;) {
            int oc[ORC_MAX_PLAYERS][2];
            uint32_t os[ORC_MAX_PLAYERS];
            REAL prod = RLIT(1.0);
            int ok = 1;
            for (int i = 0; i < k && ok; i++) {
                int p = opp[i], o = idx[i];
                int a0 = OH(c, p, o, 0), a1 = OH(c, p, o, 1);
                oc[i][0] = a0;
                oc[i][1] = a1;
                if (hc0 == a0 || hc0 == a1 || hc1 == a0 || hc1 == a1) { ok = 0; break; }
                uint32_t s = OSTR(p, o);
                if (s == 0) { ok = 0; break; }
                os[i] = s;
                prod *= OREACH(c, p, n, o);
                for (int j = 0; j < i; j++)
                    if (a0 == oc[j][0] || a0 == oc[j][1] || a1 == oc[j][0] || a1 == oc[j][1]) {
                        ok = 0;
                        break;
                    }
            }
            if (ok && prod > 0) {
                uint32_t best = hs;
                for (int i = 0; i < k; i++) if (os[i] > best) best = os[i];
                if (hs < best) {
                    val += prod * (-tb);
                } else {
                    int wins = 1;
                    for (int i = 0; i < k; i++) if (os[i] == best) wins++;
                    val += prod * (pot / (REAL)wins - tb);
                }
            }
            int j = k - 1;
            while (j >= 0) {
                if (++idx[j] < c->nh[opp[j]]) break;
                idx[j] = 0;
                j--;
            }
            if (j < 0) break;
        }
        OCFV(c, n, h) = val;
    }
#undef OSTR
}

/* bottom-up value and regret update at one decision node,
 * street_solve.cu:1138-1185 */
static void RSUF(prop_cfv)(RSUF(OrcCtx) *c, int n, int trav, int iter, REAL *regrets,
                           REAL *strategy_sum)
{
    const OrcNode *x = &c->t->nodes[n];
    if (x->type != ORC_NODE_DECISION) return;
    int na = x->num_children;
    for (int h = 0; h < c->nh[trav]; h++) {
        if (x->player == trav) {
            REAL val = 0;
            for (int a = 0; a < na; a++) {
                int ch = c->t->children[x->first_child + a];
                val += OST(c->strategy, c, n, a, h) * OCFV(c, ch, h);
            }
            OCFV(c, n, h) = val;
            for (int a = 0; a < na; a++) {
                int ch = c->t->children[x->first_child + a];
                OST(regrets, c, n, a, h) += OCFV(c, ch, h) - val;
            }
            REAL d = (REAL)iter / ((REAL)iter + RLIT(1.0));
            for (int a = 0; a < na; a++) OST(regrets, c, n, a, h) *= d;
            for (int a = 0; a < na; a++)
                OST(strategy_sum, c, n, a, h) += (REAL)iter * OST(c->strategy, c, n, a, h);
        } else {
            REAL val = 0;
            for (int a = 0; a < na; a++) {
                int ch = c->t->children[x->first_child + a];
                val += OCFV(c, ch, h);
            }
            OCFV(c, n, h) = val;
        }
    }
}

/* hand strengths per (showdown node, player, hand), street_solve.cu:513-550 */
static void RSUF(strengths)(RSUF(OrcCtx) *c, const int *sd_nodes, int nsd)
{
    for (int s = 0; s < nsd; s++) {
        const OrcNode *x = &c->t->nodes[sd_nodes[s]];
        for (int p = 0; p < c->np; p++)
            for (int h = 0; h < c->nh[p]; h++) {
                uint32_t *dst = &c->strength[((size_t)s * c->np + p) * c->max_h + h];
                if (!x->active_players[p]) { *dst = 0; continue; }
                int h0 = OH(c, p, h, 0), h1 = OH(c, p, h, 1);
                if (RSUF(board_blocked)(x, h0, h1)) { *dst = 0; continue; }
                int c7[7] = {x->board_cards[0], x->board_cards[1], x->board_cards[2],
                             x->board_cards[3], x->board_cards[4], h0, h1};
                *dst = orc_eval7(c7);
            }
    }
}

static int RSUF(ctx_init)(RSUF(OrcCtx) *c, const OrcTree *t, const int *hands,
                          const int *num_hands, int **sd_nodes_out, int *nsd_out)
{
    memset(c, 0, sizeof(*c));
    c->t = t;
    c->np = t->num_players;
    c->N = t->num_nodes;
    c->hands = hands;
    c->nh = num_hands;
    for (int p = 0; p < c->np; p++) if (num_hands[p] > c->max_h) c->max_h = num_hands[p];
    if (c->max_h == 0 || c->np == 0) return -1;
    size_t N = (size_t)c->N, H = (size_t)c->max_h;
    c->reach = (REAL *)calloc((size_t)c->np * N * H, sizeof(REAL));
    c->cfv = (REAL *)calloc(N * H, sizeof(REAL));
    c->strategy = (REAL *)calloc(N * ORC_MAX_ACTIONS * H, sizeof(REAL));
    c->sd_local = (int *)calloc(N, sizeof(int));
    int *sd = (int *)malloc((N + 1) * sizeof(int));
    int nsd = 0;
    for (int i = 0; i < c->N; i++)
        if (t->nodes[i].type == ORC_NODE_SHOWDOWN) { c->sd_local[i] = nsd; sd[nsd++] = i; }
    c->strength = (uint32_t *)calloc((size_t)(nsd ? nsd : 1) * c->np * H, sizeof(uint32_t));
    if (t->is_river && nsd > 0) RSUF(strengths)(c, sd, nsd);
    *sd_nodes_out = sd;
    *nsd_out = nsd;
    return 0;
}

static void RSUF(ctx_free)(RSUF(OrcCtx) *c)
{
    free(c->reach);
    free(c->cfv);
    free(c->strategy);
    free(c->strength);
    free(c->sd_local);
}

/* root reach of one player: weights at node 0, zero elsewhere
 * (street_solve.cu:1493-1498) */
static void RSUF(reach_root)(RSUF(OrcCtx) *c, int rp, const float *weights)
{
    REAL *r = &OREACH(c, rp, 0, 0);
    memset(r, 0, (size_t)c->N * c->max_h * sizeof(REAL));
    for (int h = 0; h < c->nh[rp]; h++) r[h] = (REAL)weights[(size_t)rp * c->max_h + h];
}

/* Card-removal aggregates of one counted opponent at one terminal: the
 * opponent's reach on each combo {x, y} (M, symmetric, zero diagonal), its
 * card sums u(x) = sum_y M[x][y] and total F = sum u / 2, over the range
 * entries that share no card with the board; cnt / cu / cF hold the same sums
 * over 0/1 entries (1 where the reach is positive), in exact integers. */
typedef struct {
    double M[52][52], u[52], F;
    long long cnt[52][52], cu[52], cF;
} RSUF(OppAgg);

static void RSUF(opp_aggregate)(RSUF(OrcCtx) *c, const OrcNode *x, int node, int p,
                                RSUF(OppAgg) *g)
{
    memset(g, 0, sizeof(*g));
    for (int o = 0; o < c->nh[p]; o++) {
        int a0 = OH(c, p, o, 0), a1 = OH(c, p, o, 1);
        if (a0 == a1 || RSUF(board_blocked)(x, a0, a1)) continue;
        double r = (double)OREACH(c, p, node, o);
        long long pos = r > 0;
        g->M[a0][a1] += r;
        g->M[a1][a0] += r;
        g->u[a0] += r;
        g->u[a1] += r;
        g->F += r;
        g->cnt[a0][a1] += pos;
        g->cnt[a1][a0] += pos;
        g->cu[a0] += pos;
        g->cu[a1] += pos;
        g->cF += pos;
    }
}

/* opp_mass for one or two counted opponents and every traverser hand of one
 * terminal at once, by inclusion-exclusion over shared cards instead of the
 * odometer (same sum: opponent hands pairwise disjoint, disjoint from the
 * traverser hand {a, b} and from the board).  With R = F - u(a) - u(b) +
 * M[a][b] (an opponent's mass avoiding {a, b}) and u'(z) = u(z) - M[z][a] -
 * M[z][b] (its card sums over hands avoiding {a, b}):
 *   one opponent:  R
 *   two opponents: R1 R2 - sum_{z not in {a,b}} u1'(z) u2'(z) + Q',
 *                  Q' = sum over combos avoiding {a, b} of M1 M2
 * (pairs sharing one card are counted once by the card sum, pairs on the
 * same combo twice, hence + Q').  FP64 throughout.  The same formulas on the
 * 0/1 entries count the contributing tuples exactly; where that count is 0
 * the mass is exactly 0, as the reference's sum of positive products is. */
static void RSUF(closed_mass)(RSUF(OrcCtx) *c, const OrcNode *x, int node, const int *opp,
                              int k, int trav, RSUF(OppAgg) *g, double *mass)
{
    for (int i = 0; i < k; i++) RSUF(opp_aggregate)(c, x, node, opp[i], &g[i]);
    double Q = 0;
    long long cQ = 0;
    if (k == 2)
        for (int y = 0; y < 52; y++)
            for (int z = y + 1; z < 52; z++) {
                Q += g[0].M[y][z] * g[1].M[y][z];
                cQ += g[0].cnt[y][z] * g[1].cnt[y][z];
            }
    for (int h = 0; h < c->nh[trav]; h++) {
        int a = OH(c, trav, h, 0), b = OH(c, trav, h, 1);
        double R[2];
        long long cR[2];
        for (int i = 0; i < k; i++) {
            R[i] = g[i].F - g[i].u[a] - g[i].u[b] + g[i].M[a][b];
            cR[i] = g[i].cF - g[i].cu[a] - g[i].cu[b] + g[i].cnt[a][b];
        }
        if (k == 1) {
            mass[h] = cR[0] == 0 ? 0.0 : R[0];
            continue;
        }
        double S = 0;
        long long cS = 0;
        for (int z = 0; z < 52; z++) {
            if (z == a || z == b) continue;
            double u1 = g[0].u[z] - g[0].M[z][a] - g[0].M[z][b];
            double u2 = g[1].u[z] - g[1].M[z][a] - g[1].M[z][b];
            S += u1 * u2;
            cS += (g[0].cu[z] - g[0].cnt[z][a] - g[0].cnt[z][b]) *
                  (g[1].cu[z] - g[1].cnt[z][a] - g[1].cnt[z][b]);
        }
        double Qab = Q, sa = 0, sb = 0;
        long long cQab = cQ, ca = 0, cb = 0;
        for (int z = 0; z < 52; z++) {
            sa += g[0].M[a][z] * g[1].M[a][z];
            sb += g[0].M[b][z] * g[1].M[b][z];
            ca += g[0].cnt[a][z] * g[1].cnt[a][z];
            cb += g[0].cnt[b][z] * g[1].cnt[b][z];
        }
        Qab = Q - sa - sb + g[0].M[a][b] * g[1].M[a][b];
        cQab = cQ - ca - cb + g[0].cnt[a][b] * g[1].cnt[a][b];
        long long cnt = cR[0] * cR[1] - cS + cQab;
        mass[h] = cnt == 0 ? 0.0 : R[0] * R[1] - S + Qab;
    }
}

/* terminal values of one traverser pass with closed forms for folds and
 * leaves with 1-2 counted opponents (the FP64 checker at sizes where the
 * odometer is out of reach); every other terminal as in terminals().
 * Terminals write disjoint value rows, so they are spread over threads. */
static void RSUF(terminals_closed)(RSUF(OrcCtx) *c, int trav, const float *leaf_values)
{
    const OrcTree *t = c->t;
    memset(c->cfv, 0, (size_t)c->N * c->max_h * sizeof(REAL));
#pragma omp parallel
    {
        RSUF(OppAgg) *g = (RSUF(OppAgg) *)malloc(2 * sizeof(RSUF(OppAgg)));
        double *mass = (double *)malloc((size_t)c->max_h * sizeof(double));
#pragma omp for schedule(dynamic, 8)
        for (int n = 0; n < c->N; n++) {
            const OrcNode *x = &t->nodes[n];
            int opp[ORC_MAX_PLAYERS], k = 0;
            if (x->type == ORC_NODE_FOLD) {
                for (int p = 0; p < c->np; p++) if (p != trav) opp[k++] = p;
                if (k > 2) { RSUF(fold_value)(c, n, trav); continue; }
                REAL payoff = (trav == x->player) ? (REAL)(x->pot - x->bets[trav])
                                                   : -(REAL)x->bets[trav];
                RSUF(closed_mass)(c, x, n, opp, k, trav, g, mass);
                for (int h = 0; h < c->nh[trav]; h++) OCFV(c, n, h) = payoff * (REAL)mass[h];
            } else if (x->type == ORC_NODE_SHOWDOWN) {
                if (t->is_river) RSUF(showdown_value)(c, n, trav);
            } else if (x->type == ORC_NODE_LEAF && leaf_values) {
                for (int p = 0; p < c->np; p++)
                    if (p != trav && x->active_players[p]) opp[k++] = p;
                if (k == 0 || k > 2 || x->leaf_idx < 0) {
                    RSUF(leaf_value)(c, n, trav, leaf_values);
                    continue;
                }
                RSUF(closed_mass)(c, x, n, opp, k, trav, g, mass);
                for (int h = 0; h < c->nh[trav]; h++) {
                    REAL ev = (REAL)leaf_values[((size_t)x->leaf_idx * c->np + trav) * c->max_h + h];
                    OCFV(c, n, h) = ev * (REAL)mass[h];
                }
            }
        }
        free(mass);
        free(g);
    }
}

static void RSUF(terminals)(RSUF(OrcCtx) *c, int trav, const float *leaf_values)
{
    const OrcTree *t = c->t;
    if (c->closed) {
        RSUF(terminals_closed)(c, trav, leaf_values);
        return;
    }
    memset(c->cfv, 0, (size_t)c->N * c->max_h * sizeof(REAL));
    /* terminals write disjoint value rows; each row is computed exactly as in
     * a serial loop, so spreading them over threads changes no bit */
#pragma omp parallel for schedule(dynamic, 4)
    for (int i = 0; i < c->N; i++) {
        int ty = t->nodes[i].type;
        if (ty == ORC_NODE_FOLD) RSUF(fold_value)(c, i, trav);
        else if (ty == ORC_NODE_SHOWDOWN && t->is_river) RSUF(showdown_value)(c, i, trav);
        else if (ty == ORC_NODE_LEAF && leaf_values) RSUF(leaf_value)(c, i, trav, leaf_values);
    }
}

static int RSUF(solve_impl)(const OrcTree *t, const int *hands, const float *weights,
                            const int *num_hands, const float *leaf_values, const int *frozen,
                            int iterations, REAL *root_strategy, REAL *root_ev,
                            REAL *avg_strategies, int *avg_node_ids, REAL *regrets_out,
                            REAL *strategy_sum_out, int closed)
{
    RSUF(OrcCtx) c;
    int *sd_nodes = NULL, nsd = 0;
    if (RSUF(ctx_init)(&c, t, hands, num_hands, &sd_nodes, &nsd) != 0) return -1;
    c.closed = closed;
    size_t N = (size_t)c.N, H = (size_t)c.max_h;
    REAL *regrets = (REAL *)calloc(N * ORC_MAX_ACTIONS * H, sizeof(REAL));
    REAL *ssum = (REAL *)calloc(N * ORC_MAX_ACTIONS * H, sizeof(REAL));
    const int *lo = t->level_order;

    for (int it = 1; it <= iterations; it++) {
        for (int trav = 0; trav < c.np; trav++) {
            for (int i = 0; i < c.N; i++) RSUF(regret_match)(&c, regrets, i);
            if (frozen)
                for (int i = 0; i < c.N; i++)
                    if (t->nodes[i].type == ORC_NODE_DECISION) RSUF(freeze)(&c, frozen, i);
            for (int rp = 0; rp < c.np; rp++) {
                if (rp == trav) continue;
                RSUF(reach_root)(&c, rp, weights);
                for (int i = 0; i < c.N; i++) RSUF(prop_reach)(&c, lo[i], rp);
            }
            RSUF(terminals)(&c, trav, leaf_values);
            for (int i = c.N - 1; i >= 0; i--) RSUF(prop_cfv)(&c, lo[i], trav, it, regrets, ssum);
        }
    }

    /* outputs, street_solve.cu:1563-1612 */
    const OrcNode *root = &t->nodes[0];
    if (root_strategy && root->player >= 0) {
        int na = root->num_children, nh = num_hands[root->player];
        for (int a = 0; a < na; a++)
            for (int h = 0; h < nh; h++)
                root_strategy[(size_t)a * nh + h] = OST(c.strategy, &c, 0, a, h);
    }
    if (root_ev)
        for (size_t h = 0; h < H; h++) root_ev[h] = c.cfv[h];
    if (avg_strategies) {
        int di = 0;
        for (int i = 0; i < c.N; i++) {
            const OrcNode *x = &t->nodes[i];
            if (x->type != ORC_NODE_DECISION) continue;
            if (avg_node_ids) avg_node_ids[di] = i;
            REAL *dst = &avg_strategies[(size_t)di * ORC_MAX_ACTIONS * H];
            for (size_t z = 0; z < ORC_MAX_ACTIONS * H; z++) dst[z] = 0;
            int p = x->player;
            if (p >= 0 && p < c.np) {
                int na = x->num_children;
                for (int h = 0; h < num_hands[p]; h++) {
                    REAL sum = 0;
                    for (int a = 0; a < na; a++) {
                        REAL v = OST(ssum, &c, i, a, h);
                        if (v < 0) v = 0;
                        sum += v;
                    }
                    REAL inv = (sum > 0) ? (RLIT(1.0) / sum) : (RLIT(1.0) / (REAL)na);
                    for (int a = 0; a < na; a++) {
                        REAL v = OST(ssum, &c, i, a, h);
                        if (v < 0) v = 0;
                        dst[(size_t)a * H + h] = (sum > 0) ? (v * inv) : inv;
                    }
                }
            }
            di++;
        }
    }
    if (regrets_out) memcpy(regrets_out, regrets, N * ORC_MAX_ACTIONS * H * sizeof(REAL));
    if (strategy_sum_out) memcpy(strategy_sum_out, ssum, N * ORC_MAX_ACTIONS * H * sizeof(REAL));
    free(regrets);
    free(ssum);
    free(sd_nodes);
    RSUF(ctx_free)(&c);
    return 0;
}

int RSUF(orc_solve)(const OrcTree *t, const int *hands, const float *weights,
                    const int *num_hands, const float *leaf_values, const int *frozen,
                    int iterations, REAL *root_strategy, REAL *root_ev,
                    REAL *avg_strategies, int *avg_node_ids, REAL *regrets_out,
                    REAL *strategy_sum_out)
{
    return RSUF(solve_impl)(t, hands, weights, num_hands, leaf_values, frozen, iterations,
                            root_strategy, root_ev, avg_strategies, avg_node_ids, regrets_out,
                            strategy_sum_out, 0);
}

#undef OH
#undef OREACH
#undef OCFV
#undef OST
