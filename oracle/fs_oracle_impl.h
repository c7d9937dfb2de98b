/*
 * fs_oracle_impl.h -- CFR body of the multi-street oracle, included twice by
 * fs_oracle.c (REAL = float: the reference's arithmetic and order; REAL =
 * double).  TEST INFRASTRUCTURE ONLY.
 *
 * fso_solve_*: hands [2][200][2], weights [2][200] (the FSTreeData layout),
 * nh[2]; node_depth / max_depth as fs_build_tree writes them.  Outputs (any
 * may be NULL): root_strategy [na_root][nh_root] (the last regret-matched
 * strategy at node 0), avg [N][6][max_h] (normalised strategy sums at
 * decision nodes, 0 elsewhere), cfv [N][max_h] (the last traverser's
 * values); snap_root [n_snap][na_root][nh_root]: the root strategy after
 * iteration snap_iters[j] (the same read-out as root_strategy, taken on the
 * way).  Loops over the nodes of one level (and over all nodes where each
 * writes only its own rows) run on OpenMP threads: no sums cross threads, so
 * the results do not depend on the thread count.  Returns 0, or -1 on bad
 * input.
 */

int FSUF(fso_solve)(const FsoNode *nodes, const int *children, int N, const int *node_depth, int max_depth,
                    const int *hands, const float *weights, const int *nh, int iterations, REAL *root_strategy,
                    REAL *avg, REAL *cfv_out, int n_snap, const int *snap_iters, REAL *snap_root)
{
    const int max_h = nh[0] > nh[1] ? nh[0] : nh[1];
    if (max_h <= 0 || N <= 0) return -1;
    const size_t H = (size_t)max_h, A = FSO_MAX_ACTIONS;
    REAL *regrets = (REAL *)calloc((size_t)N * A * H, sizeof(REAL));
    REAL *strategy = (REAL *)calloc((size_t)N * A * H, sizeof(REAL));
    REAL *ssum = (REAL *)calloc((size_t)N * A * H, sizeof(REAL));
    REAL *reach = (REAL *)calloc((size_t)N * H, sizeof(REAL));
    REAL *cfv = (REAL *)calloc((size_t)N * H, sizeof(REAL));
    /* levels: nodes by BFS depth, in index order within a level (:1055-1064) */
    int *lev_off = (int *)calloc((size_t)max_depth + 2, sizeof(int));
    int *lev = (int *)malloc((size_t)N * sizeof(int));
    for (int i = 0; i < N; i++) lev_off[node_depth[i] + 1]++;
    for (int d = 0; d <= max_depth; d++) lev_off[d + 1] += lev_off[d];
    {
        int *fill = (int *)calloc((size_t)max_depth + 1, sizeof(int));
        for (int i = 0; i < N; i++) lev[lev_off[node_depth[i]] + fill[node_depth[i]]++] = i;
        free(fill);
    }
    /* strengths per (showdown node, player, hand), :366-399 */
    uint32_t *str = (uint32_t *)calloc((size_t)N * 2 * H, sizeof(uint32_t));
#pragma omp parallel for schedule(dynamic, 256)
    for (int x = 0; x < N; x++) {
        if (nodes[x].type != 2) continue;
        for (int p = 0; p < 2; p++)
            for (int h = 0; h < nh[p]; h++) {
                int c0 = hands[(p * FSO_MAX_HANDS + h) * 2], c1 = hands[(p * FSO_MAX_HANDS + h) * 2 + 1];
                int blocked = 0;
                for (int b = 0; b < nodes[x].num_board; b++)
                    if (c0 == nodes[x].board_cards[b] || c1 == nodes[x].board_cards[b]) blocked = 1;
                if (!blocked) {
                    int c7[7] = {nodes[x].board_cards[0], nodes[x].board_cards[1], nodes[x].board_cards[2],
                                 nodes[x].board_cards[3], nodes[x].board_cards[4], c0, c1};
                    str[((size_t)x * 2 + p) * H + h] = orc_eval7(c7);
                }
            }
    }
    const REAL half_start = (REAL)nodes[0].pot * FLIT(0.5);
#define ST(arr, n, a, h) (arr)[((size_t)(n) * A + (a)) * H + (h)]
#define HC(p, i, k) hands[((p) * FSO_MAX_HANDS + (i)) * 2 + (k)]
    for (int it = 1; it <= iterations; it++) {
        for (int trav = 0; trav < 2; trav++) {
            const int opp = 1 - trav;
            /* regret matching, :652-684 */
#pragma omp parallel for schedule(dynamic, 1024)
            for (int x = 0; x < N; x++) {
                const FsoNode *n = &nodes[x];
                if (n->type != 0) continue;
                const int na = n->num_children;
                for (int h = 0; h < nh[n->player]; h++) {
                    REAL sum = 0;
                    for (int a = 0; a < na; a++) {
                        REAL r = ST(regrets, x, a, h);
                        sum += r > 0 ? r : 0;
                    }
                    const REAL inv = sum > 0 ? FLIT(1.0) / sum : 0;
                    for (int a = 0; a < na; a++) {
                        REAL r = ST(regrets, x, a, h);
                        ST(strategy, x, a, h) = sum > 0 ? (r > 0 ? r : 0) * inv : FLIT(1.0) / (REAL)na;
                    }
                }
            }
            /* the opponent's reach, :686-729 */
            memset(reach, 0, (size_t)N * H * sizeof(REAL));
            for (int h = 0; h < nh[opp]; h++) reach[h] = (REAL)weights[opp * FSO_MAX_HANDS + h];
            for (int d = 0; d <= max_depth; d++)
#pragma omp parallel for schedule(dynamic, 256)
                for (int k = lev_off[d]; k < lev_off[d + 1]; k++) {
                    const int x = lev[k];
                    const FsoNode *n = &nodes[x];
                    if (n->type != 0 && n->type != 3) continue;
                    for (int h = 0; h < nh[opp]; h++) {
                        const REAL pr = reach[(size_t)x * H + h];
                        for (int a = 0; a < n->num_children; a++) {
                            const int c = children[n->first_child + a];
                            reach[(size_t)c * H + h] =
                                (n->type == 0 && n->player == opp) ? pr * ST(strategy, x, a, h) : pr;
                        }
                    }
                }
            /* terminal values, :731-833 */
            memset(cfv, 0, (size_t)N * H * sizeof(REAL));
#pragma omp parallel for schedule(dynamic, 256)
            for (int x = 0; x < N; x++) {
                const FsoNode *n = &nodes[x];
                if (n->type != 1 && n->type != 2) continue;
                for (int h = 0; h < nh[trav]; h++) {
                    const int hc0 = HC(trav, h, 0), hc1 = HC(trav, h, 1);
                    REAL v = 0;
                    if (n->type == 1) {
                        const int winner = n->player, loser = 1 - winner;
                        const REAL payoff = trav == winner ? half_start + (REAL)n->bets[loser]
                                                           : -(half_start + (REAL)n->bets[trav]);
                        REAL s = 0;
                        for (int o = 0; o < nh[opp]; o++) {
                            const int oc0 = HC(opp, o, 0), oc1 = HC(opp, o, 1);
                            if (hc0 == oc0 || hc0 == oc1 || hc1 == oc0 || hc1 == oc1) continue;
                            int blocked = 0;
                            for (int b = 0; b < n->num_board; b++)
                                if (oc0 == n->board_cards[b] || oc1 == n->board_cards[b]) blocked = 1;
                            if (blocked) continue;
                            s += reach[(size_t)x * H + o];
                        }
                        v = s * payoff;
                    } else {
                        const uint32_t hs = str[((size_t)x * 2 + trav) * H + h];
                        if (hs != 0) {
                            const REAL half_pot = (REAL)n->pot * FLIT(0.5);
                            for (int o = 0; o < nh[opp]; o++) {
                                const int oc0 = HC(opp, o, 0), oc1 = HC(opp, o, 1);
                                if (hc0 == oc0 || hc0 == oc1 || hc1 == oc0 || hc1 == oc1) continue;
                                const uint32_t os = str[((size_t)x * 2 + opp) * H + o];
                                if (os == 0) continue;
                                const REAL w = reach[(size_t)x * H + o];
                                if (hs > os) v = FMA(w, half_pot, v);
                                else if (hs < os) v = FMA(-w, half_pot, v);
                            }
                        }
                    }
                    cfv[(size_t)x * H + h] = v;
                }
            }
            /* values bottom-up, regrets and strategy sums, :835-892 */
            const REAL disc = (REAL)it / ((REAL)it + FLIT(1.0));
            for (int d = max_depth; d >= 0; d--)
#pragma omp parallel for schedule(dynamic, 256)
                for (int k = lev_off[d]; k < lev_off[d + 1]; k++) {
                    const int x = lev[k];
                    const FsoNode *n = &nodes[x];
                    if (n->type != 0 && n->type != 3) continue;
                    const int na = n->num_children;
                    for (int h = 0; h < nh[trav]; h++) {
                        REAL v = 0;
                        if (n->type == 0 && n->player == trav) {
                            for (int a = 0; a < na; a++)
                                v = FMA(ST(strategy, x, a, h), cfv[(size_t)children[n->first_child + a] * H + h], v);
                            cfv[(size_t)x * H + h] = v;
                            for (int a = 0; a < na; a++)
                                ST(regrets, x, a, h) += cfv[(size_t)children[n->first_child + a] * H + h] - v;
                            for (int a = 0; a < na; a++) ST(regrets, x, a, h) *= disc;
                            for (int a = 0; a < na; a++)
                                ST(ssum, x, a, h) = FMA((REAL)it, ST(strategy, x, a, h), ST(ssum, x, a, h));
                        } else {
                            for (int a = 0; a < na; a++) v += cfv[(size_t)children[n->first_child + a] * H + h];
                            if (n->type == 3) v = v / (REAL)na;
                            cfv[(size_t)x * H + h] = v;
                        }
                    }
                }
        }
        for (int j = 0; j < n_snap; j++)
            if (snap_iters[j] == it) {
                const int rp = nodes[0].player, na = nodes[0].num_children;
                REAL *dst = snap_root + (size_t)j * na * nh[rp];
                for (int a = 0; a < na; a++)
                    for (int h = 0; h < nh[rp]; h++) dst[(size_t)a * nh[rp] + h] = ST(strategy, 0, a, h);
            }
    }
    if (root_strategy) {
        const int rp = nodes[0].player, na = nodes[0].num_children;
        for (int a = 0; a < na; a++)
            for (int h = 0; h < nh[rp]; h++) root_strategy[(size_t)a * nh[rp] + h] = ST(strategy, 0, a, h);
    }
    if (avg) {
        /* :1516-1540 */
        memset(avg, 0, (size_t)N * A * H * sizeof(REAL));
#pragma omp parallel for schedule(dynamic, 1024)
        for (int x = 0; x < N; x++) {
            const FsoNode *n = &nodes[x];
            if (n->type != 0) continue;
            const int na = n->num_children;
            for (int h = 0; h < nh[n->player]; h++) {
                REAL sum = 0;
                for (int a = 0; a < na; a++) {
                    REAL s = ST(ssum, x, a, h);
                    sum += s > 0 ? s : 0;
                }
                const REAL inv = sum > 0 ? FLIT(1.0) / sum : 0;
                for (int a = 0; a < na; a++) {
                    REAL s = ST(ssum, x, a, h);
                    ST(avg, x, a, h) = sum > 0 ? (s > 0 ? s * inv : 0) : FLIT(1.0) / (REAL)na;
                }
            }
        }
    }
    if (cfv_out) memcpy(cfv_out, cfv, (size_t)N * H * sizeof(REAL));
#undef ST
#undef HC
    free(regrets);
    free(strategy);
    free(ssum);
    free(reach);
    free(cfv);
    free(lev_off);
    free(lev);
    free(str);
    return 0;
}
