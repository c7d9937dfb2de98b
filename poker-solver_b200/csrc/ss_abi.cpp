// ss_abi.cpp -- the exported C ABI (include/street_solve.h).
//
// Compiled once per SS_MAX_HANDS (200: the reference layout of SSTreeData,
// 1326: every 2-card combo); everything else lives in the engine, which only
// sees plain pointers.
#include "street_solve.h"

#include "ss_engine.h"
#include "ss_leaf.h"

#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

namespace {

template <class T>
T *copy_out(const std::vector<T> &v, size_t extra = 0) {
    T *p = static_cast<T *>(std::malloc((v.size() + extra) * sizeof(T) + 1));
    if (p && !v.empty()) std::memcpy(p, v.data(), v.size() * sizeof(T));
    return p;
}

int to_problem(const SSTreeData *td, ssb::Problem *pb) {
    if (!td || !td->nodes || !td->children) {
        ssb::set_error("tree_data has no nodes (call ss_build_tree first)");
        return SS_ERR_INVALID;
    }
    if (td->num_players < 1 || td->num_players > SS_MAX_PLAYERS) {
        ssb::set_error("num_players must be 1..6");
        return SS_ERR_INVALID;
    }
    pb->nodes = td->nodes;
    pb->children = td->children;
    pb->num_nodes = td->num_nodes;
    pb->num_children_total = td->num_children_total;
    pb->num_players = td->num_players;
    for (int p = 0; p < td->num_players; ++p) {
        if (td->num_hands[p] < 0 || td->num_hands[p] > SS_MAX_HANDS) {
            ssb::set_error("num_hands exceeds SS_MAX_HANDS of this build (see ss_abi_info)");
            return SS_ERR_INVALID;
        }
        pb->hands[p] = &td->hands[p][0][0];
        pb->weights[p] = td->weights[p];
        pb->num_hands[p] = td->num_hands[p];
    }
    for (int i = 0; i < SS_MAX_BOARD; ++i) pb->board[i] = td->board[i];
    pb->num_board = td->num_board;
    pb->leaf_values = td->leaf_values;
    pb->num_leaves = td->num_leaves;
    pb->frozen = td->frozen_action;
    pb->starting_pot = td->starting_pot;
    pb->is_river = td->is_river;
    return SS_OK;
}

}  // namespace

struct SSSession {
    ssb::Session *impl;
};

struct SSServer {
    ssb::Server *impl;
};

extern "C" {

int ss_build_tree_ex(const int *board, int num_board, int starting_pot, int effective_stack,
                     const float *bet_sizes, int num_bet_sizes, int num_players,
                     const int *acting_order, int is_river, int use_cont_strats, int max_raises,
                     SSTreeData *tree_out) {
    if (!tree_out) {
        ssb::set_error("tree_out is NULL");
        return SS_ERR_INVALID;
    }
    std::memset(tree_out, 0, sizeof(SSTreeData));
    ssb::BuiltTree bt;
    int rc;
    try {
        rc = ssb::build_street_tree(board, num_board, starting_pot, effective_stack, bet_sizes,
                                    num_bet_sizes, num_players, acting_order, is_river,
                                    use_cont_strats, max_raises, &bt);
    } catch (const std::bad_alloc &) {
        ssb::set_error("out of host memory while building the tree");
        return SS_ERR_NOMEM;
    }
    if (rc != SS_OK) return rc;
    const int n = static_cast<int>(bt.nodes.size());
    std::vector<int> lists[4];
    for (int i = 0; i < n; ++i) {
        switch (bt.nodes[i].type) {
            case SS_NODE_DECISION: lists[0].push_back(i); break;
            case SS_NODE_SHOWDOWN: lists[1].push_back(i); break;
            case SS_NODE_LEAF: lists[2].push_back(i); break;
            case SS_NODE_FOLD: lists[3].push_back(i); break;
            default: break;
        }
    }
    SSTreeData &t = *tree_out;
    t.nodes = copy_out(bt.nodes);
    t.children = copy_out(bt.children);
    t.level_order = copy_out(bt.level_order);
    t.node_depth = copy_out(bt.node_depth);
    t.decision_node_indices = copy_out(lists[0], 1);
    t.showdown_node_indices = copy_out(lists[1], 1);
    t.leaf_node_indices = copy_out(lists[2], 1);
    t.fold_node_indices = copy_out(lists[3], 1);
    if (!t.nodes || !t.children || !t.level_order || !t.node_depth || !t.decision_node_indices ||
        !t.showdown_node_indices || !t.leaf_node_indices || !t.fold_node_indices) {
        ss_free_tree(tree_out);
        ssb::set_error("out of host memory while building the tree");
        return SS_ERR_NOMEM;
    }
    t.num_nodes = n;
    t.num_children_total = static_cast<int>(bt.children.size());
    t.num_leaves = bt.num_leaves;
    t.max_depth = bt.max_depth;
    t.num_decision_nodes = static_cast<int>(lists[0].size());
    t.num_showdown_nodes = static_cast<int>(lists[1].size());
    t.num_leaf_nodes = static_cast<int>(lists[2].size());
    t.num_fold_nodes = static_cast<int>(lists[3].size());
    t.is_river = is_river;
    t.starting_pot = starting_pot;
    t.effective_stack = effective_stack;
    t.num_players = num_players;
    for (int i = 0; i < num_board && i < SS_MAX_BOARD; ++i) t.board[i] = board[i];
    t.num_board = num_board;
    return SS_OK;
}

int ss_build_tree(const int *board, int num_board, int starting_pot, int effective_stack,
                  const float *bet_sizes, int num_bet_sizes, int num_players,
                  const int *acting_order, int is_river, int use_cont_strats, SSTreeData *tree_out) {
    return ss_build_tree_ex(board, num_board, starting_pot, effective_stack, bet_sizes,
                            num_bet_sizes, num_players, acting_order, is_river, use_cont_strats,
                            SS_MAX_RAISES, tree_out);
}

void ss_free_tree(SSTreeData *td) {
    if (!td) return;
    std::free(td->nodes);
    std::free(td->children);
    std::free(td->level_order);
    std::free(td->node_depth);
    std::free(td->decision_node_indices);
    std::free(td->showdown_node_indices);
    std::free(td->leaf_node_indices);
    std::free(td->fold_node_indices);
    std::memset(td, 0, sizeof(SSTreeData));
}

void ss_free_output(SSOutput *out) {
    if (!out) return;
    std::free(out->root_strategy);
    std::free(out->root_ev);
    if (!ssb::host_block_give(out->avg_strategies)) std::free(out->avg_strategies);
    std::free(out->avg_strategy_node_ids);
    std::memset(out, 0, sizeof(SSOutput));
}

void ss_default_options(SSSolveOptions *o) {
    if (!o) return;
    o->device = 0;
    o->graph_iterations = 10;
    o->target_exploitability = -1.f;
    o->check_every = 50;
    o->compute_exploitability = 0;
}

int ss_solve_gpu_ex(SSTreeData *td, int max_iterations, const SSSolveOptions *opts,
                    SSOutput *output, SSSolveStats *stats) {
    if (!output) {
        ssb::set_error("output is NULL");
        return SS_ERR_INVALID;
    }
    std::memset(output, 0, sizeof(SSOutput));
    ssb::Problem pb;
    int rc = to_problem(td, &pb);
    if (rc != SS_OK) return rc;
    SSSolveOptions o;
    ss_default_options(&o);
    if (opts) o = *opts;
    ssb::SolveConfig cfg;
    cfg.device = o.device;
    cfg.graph_iterations = o.graph_iterations;
    cfg.target_exploitability = o.target_exploitability;
    cfg.check_every = o.check_every;
    cfg.compute_exploitability = o.compute_exploitability;
    try {
        return ssb::solve(pb, max_iterations, cfg, output, stats);
    } catch (const std::bad_alloc &) {
        ssb::set_error("out of host memory");
        return SS_ERR_NOMEM;
    }
}

int ss_solve_gpu(SSTreeData *td, int max_iterations, SSOutput *output) {
    return ss_solve_gpu_ex(td, max_iterations, nullptr, output, nullptr);
}

int ss_solve_gpu_noalloc(SSTreeData *td, int max_iterations, SSOutput *output) {
    ssb::Problem pb;
    int rc = to_problem(td, &pb);
    if (rc != SS_OK) return rc;
    try {
        return ssb::solve_noalloc(pb, max_iterations, output);
    } catch (const std::bad_alloc &) {
        ssb::set_error("out of host memory");
        return SS_ERR_NOMEM;
    }
}

int ss_exploitability_gpu(const SSTreeData *td, const float *avg, double *expl_pct,
                          double *nashconv, double *br_value, double *cur_value,
                          double *deal_mass) {
    ssb::Problem pb;
    int rc = to_problem(td, &pb);
    if (rc != SS_OK) return rc;
    if (!avg) {
        ssb::set_error("avg_strategies is NULL");
        return SS_ERR_INVALID;
    }
    try {
        return ssb::exploitability(pb, avg, expl_pct, nashconv, br_value, cur_value, deal_mass);
    } catch (const std::bad_alloc &) {
        ssb::set_error("out of host memory");
        return SS_ERR_NOMEM;
    }
}

int ss_abi_info(SSAbiInfo *info) {
    if (!info) return SS_ERR_INVALID;
    info->abi_version = 1;
    info->max_hands = SS_MAX_HANDS;
    info->max_players = SS_MAX_PLAYERS;
    info->max_actions = SS_MAX_ACTIONS;
    info->sizeof_node = static_cast<int>(sizeof(SSNode));
    info->sizeof_tree = static_cast<int>(sizeof(SSTreeData));
    info->sizeof_output = static_cast<int>(sizeof(SSOutput));
    return SS_OK;
}

int ss_session_create(const SSTreeData *td, const SSSolveOptions *opts, SSSession **out) {
    if (!out) {
        ssb::set_error("out is NULL");
        return SS_ERR_INVALID;
    }
    *out = nullptr;
    ssb::Problem pb;
    int rc = to_problem(td, &pb);
    if (rc != SS_OK) return rc;
    SSSolveOptions o;
    ss_default_options(&o);
    if (opts) o = *opts;
    ssb::SolveConfig cfg;
    cfg.device = o.device;
    cfg.graph_iterations = o.graph_iterations;
    cfg.target_exploitability = o.target_exploitability;
    cfg.check_every = o.check_every;
    cfg.compute_exploitability = o.compute_exploitability;
    try {
        ssb::Session *s = nullptr;
        rc = ssb::session_create(pb, cfg, &s);
        if (rc != SS_OK) return rc;
        *out = new SSSession{s};
        return SS_OK;
    } catch (const std::bad_alloc &) {
        ssb::set_error("out of host memory");
        return SS_ERR_NOMEM;
    }
}

int ss_session_run(SSSession *s, int iterations) {
    if (!s) return SS_ERR_INVALID;
    return ssb::session_run(s->impl, iterations);
}

int ss_session_synchronize(SSSession *s) {
    if (!s) return SS_ERR_INVALID;
    return ssb::session_sync(s->impl);
}

int ss_session_reset(SSSession *s) {
    if (!s) return SS_ERR_INVALID;
    return ssb::session_reset(s->impl);
}

int ss_session_iterations(const SSSession *s) { return s ? ssb::session_iterations(s->impl) : -1; }

int ss_session_output(SSSession *s, SSOutput *out) {
    if (!s || !out) return SS_ERR_INVALID;
    try {
        return ssb::session_output(s->impl, out);
    } catch (const std::bad_alloc &) {
        ssb::set_error("out of host memory");
        return SS_ERR_NOMEM;
    }
}

int ss_session_profile(SSSession *s, SSKernelProfile *prof) {
    if (!s || !prof) return SS_ERR_INVALID;
    return ssb::session_profile(s->impl, prof);
}

int ss_session_profile_launches(SSSession *s, SSLaunchRecord *records, int max_records, int *num_records) {
    if (!s || max_records < 0 || (max_records > 0 && !records)) return SS_ERR_INVALID;
    return ssb::session_profile_launches(s->impl, records, max_records, num_records);
}

int ss_session_exploitability(SSSession *s, double *pct, double *nash, double *br, double *cur,
                              double *z) {
    if (!s) return SS_ERR_INVALID;
    return ssb::session_exploitability(s->impl, nullptr, pct, nash, br, cur, z);
}

int ss_session_narrow(SSSession *s, int player, int node, unsigned int action_mask, int num_hands,
                      const int *hand_cards, double *weights, int *applied) {
    if (!s) return SS_ERR_INVALID;
    return ssb::session_narrow(s->impl, player, node, action_mask, num_hands, hand_cards, weights, applied);
}

void *ss_session_stream(SSSession *s) { return s ? ssb::session_stream(s->impl) : nullptr; }

void ss_session_destroy(SSSession *s) {
    if (!s) return;
    ssb::session_destroy(s->impl);
    delete s;
}

int ss_rank7_batch(const int *cards7, int n, unsigned int *strength_out) {
    return ssb::rank7_batch(cards7, n, strength_out);
}

int ss_rank7_checksum(unsigned long long *checksum, unsigned long long *category_counts) {
    if (!checksum) return SS_ERR_INVALID;
    return ssb::rank7_checksum(checksum, category_counts);
}

int ss_batch_solve(SSTreeData *const *trees, int n, int max_iterations, const SSSolveOptions *opts,
                   SSOutput *outputs, SSSolveStats *stats) {
    if (!trees || !outputs || n < 0) {
        ssb::set_error("ss_batch_solve: bad arguments");
        return SS_ERR_INVALID;
    }
    try {
        std::vector<ssb::Problem> pbs(n);
        for (int i = 0; i < n; ++i) {
            int rc = to_problem(trees[i], &pbs[i]);
            if (rc != SS_OK) return rc;
        }
        SSSolveOptions o;
        ss_default_options(&o);
        if (opts) o = *opts;
        ssb::SolveConfig cfg;
        cfg.device = o.device;
        cfg.graph_iterations = o.graph_iterations;
        cfg.target_exploitability = o.target_exploitability;
        cfg.check_every = o.check_every;
        cfg.compute_exploitability = o.compute_exploitability;
        return ssb::batch_solve(pbs, max_iterations, cfg, outputs, stats);
    } catch (const std::bad_alloc &) {
        ssb::set_error("out of host memory");
        return SS_ERR_NOMEM;
    }
}

void ss_server_default_options(SSServerOptions *o) {
    if (!o) return;
    o->device = 0;
    o->memory_budget_gb = 40.0;
    o->block_iterations = 25;
    o->target_exploitability = 0.5f;
    o->max_iterations = 1000;
    o->graph_iterations = 25;
}

int ss_server_create(const SSServerOptions *opts, SSServer **out) {
    if (!out) return SS_ERR_INVALID;
    *out = nullptr;
    SSServerOptions o;
    ss_server_default_options(&o);
    if (opts) o = *opts;
    try {
        ssb::Server *s = nullptr;
        int rc = ssb::server_create(o, &s);
        if (rc != SS_OK) return rc;
        *out = new SSServer{s};
        return SS_OK;
    } catch (const std::exception &) {
        ssb::set_error("could not start the server");
        return SS_ERR_NOMEM;
    }
}

int ss_server_submit(SSServer *s, const SSTreeData *td, long long *id) {
    if (!s || !id) return SS_ERR_INVALID;
    ssb::Problem pb;
    int rc = to_problem(td, &pb);
    if (rc != SS_OK) return rc;
    try {
        return ssb::server_submit(s->impl, pb, id);
    } catch (const std::bad_alloc &) {
        ssb::set_error("out of host memory");
        return SS_ERR_NOMEM;
    }
}

int ss_server_poll(SSServer *s, long long id, SSOutput *out, SSSolveStats *stats, double *latency_ms) {
    if (!s) return SS_ERR_INVALID;
    return ssb::server_poll(s->impl, id, out, stats, latency_ms, 0);
}

int ss_server_progress(SSServer *s, long long id, int *state, int *iterations_run) {
    if (!s) return SS_ERR_INVALID;
    return ssb::server_progress(s->impl, id, state, iterations_run);
}

int ss_server_wait(SSServer *s, long long id, SSOutput *out, SSSolveStats *stats, double *latency_ms) {
    if (!s) return SS_ERR_INVALID;
    return ssb::server_poll(s->impl, id, out, stats, latency_ms, 1);
}

void ss_server_destroy(SSServer *s) {
    if (!s) return;
    ssb::server_destroy(s->impl);
    delete s;
}

int ss_leaf_values_gpu(const SSLeafValueInput *input, float *leaf_values) {
    try {
        return ssb::leaf::leaf_values_gpu(input, leaf_values);
    } catch (const std::bad_alloc &) {
        ssb::set_error("ss_leaf_values_gpu: host allocation failed");
        return SS_ERR_NOMEM;
    }
}

int ss_leaf_opponent_tuples(int num_opponents, const int *list_sizes, int *tuples, int max_tuples) {
    if (num_opponents < 1 || num_opponents > SS_MAX_PLAYERS - 1 || !list_sizes || max_tuples < 0 ||
        (max_tuples > 0 && !tuples)) {
        ssb::set_error("ss_leaf_opponent_tuples: bad arguments");
        return SS_ERR_INVALID;
    }
    for (int k = 0; k < num_opponents; ++k)
        if (list_sizes[k] < 0 || list_sizes[k] > ssb::leaf::kMaxHands) {
            ssb::set_error("ss_leaf_opponent_tuples: list sizes must be 0..1326");
            return SS_ERR_INVALID;
        }
    try {
        std::vector<int> pos;
        const int n = ssb::leaf::opponent_tuples(num_opponents, list_sizes, &pos);
        if (n > max_tuples) {
            ssb::set_error("ss_leaf_opponent_tuples: " + std::to_string(n) + " tuples, room for " +
                           std::to_string(max_tuples));
            return SS_ERR_INVALID;
        }
        if (!pos.empty()) std::memcpy(tuples, pos.data(), pos.size() * sizeof(int));
        return n;
    } catch (const std::bad_alloc &) {
        ssb::set_error("ss_leaf_opponent_tuples: host allocation failed");
        return SS_ERR_NOMEM;
    }
}

const char *ss_last_error(void) { return ssb::last_error(); }

}  // extern "C"
