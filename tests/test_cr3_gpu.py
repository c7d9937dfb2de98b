"""Terminals with three counted opponents (4-player subgames) through the
closed forms -- folds and leaves in k_term_cr3, four-way showdowns in
k_term_sd3 (ranges of at least 16 hands route there; smaller ones
enumerate) -- on the GPU against the oracle:
* a 4-player river (125 nodes; 18 and 24 hands, a repeated combo in one
  range that keeps some terminals on enumeration, a royal-flush board where
  every showdown splits): the solver against the FP32 oracle at the strict
  tolerances of the parity tests;
* a 4-player turn with continuation leaves (5,681 nodes, 16 hands): folds
  and leaves with three counted opponents, against the FP32 oracle;
* the FP64 best response, whose 4-player deal mass also takes the closed
  form, against the oracle's FP64 CPU best response to 1e-9 relative;
* what remains on exact enumeration: the 6-player river benchmark tree
  (19,579 nodes; folds with five counted opponents, 2- to 6-way showdowns)
  at 5 hands per player, against the FP32 oracle.
The closed form itself is checked against enumeration on the host
(tests/test_cr3_host.py).  Collected after the solver's other GPU tests
(tests/conftest.py)."""
import numpy as np
import pytest

import workloads as wl
from cards import card_to_int
from test_exploitability_gpu import gpu_exploitability
from test_parity_gpu import solve, strict

pytestmark = pytest.mark.gpu


def four_player(name, seed, hands, dup_player=None):
    cfg = wl.config(name, seed=seed, num_hands=hands, num_players=4, bet_sizes=[1.0], max_raises=1)
    cfg["hands"], cfg["weights"] = wl.make_ranges(np.random.default_rng(seed), cfg["board"], 4, hands)
    if dup_player is not None:   # repeat one combo: that player's terminals keep the enumeration path
        h = cfg["hands"][dup_player].copy()
        h[1] = h[0]
        cfg["hands"][dup_player] = h
    return cfg


def oracle_f32(oracle, cfg, iters, lv):
    tree = oracle.build_tree(cfg["board"], cfg["pot"], cfg["stack"], cfg["bet_sizes"], cfg["num_players"],
                             max_raises=cfg["max_raises"])
    H, W, nh = wl.padded(cfg)
    return oracle.solve(tree, H, W, nh, iters, leaf_values=lv, precision="f32")


@pytest.mark.parametrize("seed,hands,iters,dup", [(21, 18, 6, None), (22, 24, 4, None), (23, 20, 4, 1)])
def test_four_player_river(oracle, seed, hands, iters, dup):
    cfg = four_player("river6", seed, hands, dup)
    ours, lv = solve(cfg, iters)
    strict(ours, oracle_f32(oracle, cfg, iters, lv))


def test_four_player_river_every_hand_ties(oracle):
    # a royal flush on the board: every showdown is a split of all live players
    cfg = wl.config("river6", seed=26, num_hands=18, num_players=4, bet_sizes=[1.0], max_raises=1)
    cfg["board"] = [card_to_int(x) for x in ("Ts", "Js", "Qs", "Ks", "As")]
    cfg["hands"], cfg["weights"] = wl.make_ranges(np.random.default_rng(26), cfg["board"], 4, 18)
    ours, lv = solve(cfg, 4)
    strict(ours, oracle_f32(oracle, cfg, 4, lv))


def test_four_player_turn_with_leaves(oracle):
    cfg = four_player("turn3", 24, 16)
    ours, lv = solve(cfg, 2)
    strict(ours, oracle_f32(oracle, cfg, 2, lv))


def test_four_player_best_response(oracle):
    cfg = four_player("river6", 25, 18)
    sg = wl.AbiSubgame(cfg)
    try:
        rc, out = sg.solve(5)
        assert rc == 0, wl.ssg.last_error(sg.lib)
        g = gpu_exploitability(sg, out["avg_strategies"])
    finally:
        sg.free()
    tree = oracle.build_tree(cfg["board"], cfg["pot"], cfg["stack"], cfg["bet_sizes"], 4,
                             max_raises=cfg["max_raises"])
    H, W, n = wl.padded(cfg)
    ref = oracle.exploitability(tree, H, W, n, out["avg_strategies"])
    assert abs(g["deal_mass"] - ref["deal_mass"]) <= 1e-9 * abs(ref["deal_mass"])
    for p in range(4):
        scale = max(abs(ref["br_value"][p]), abs(ref["cur_value"][p]), 1e-300)
        assert abs(g["br"][p] - ref["br_value"][p]) / scale <= 1e-9
        assert abs(g["cur"][p] - ref["cur_value"][p]) / scale <= 1e-9


def test_six_player_river_tree_small_ranges(oracle):
    cfg = wl.config("river6", seed=31, num_hands=5)
    cfg["hands"], cfg["weights"] = wl.make_ranges(np.random.default_rng(31), cfg["board"], 6, 5)
    ours, lv = solve(cfg, 3)
    strict(ours, oracle_f32(oracle, cfg, 3, lv))
