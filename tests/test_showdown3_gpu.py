"""Three-way showdowns on the river: the rank-order sweep (k_term_sd2) against
the oracle's tuple enumeration (street_solve.cu:936-1002), including boards
where many or all hands tie, and the full-size 3-player river, which the
enumeration cannot reach.  Tolerances as in test_parity_gpu."""
import numpy as np
import pytest

import workloads as wl
from cards import card_to_int
from test_exploitability_gpu import gpu_exploitability
from test_parity_gpu import diffs, oracle_pair, solve, strict


def river3(seed, nh, board=None, **over):
    cfg = wl.config("river6", seed=seed, num_players=3, **over)
    if board is not None:
        cfg["board"] = [card_to_int(c) for c in board]
    cfg["hands"], cfg["weights"] = wl.make_ranges(np.random.default_rng(seed), cfg["board"], 3, nh)
    return cfg


@pytest.mark.gpu
@pytest.mark.parametrize("seed,nh,iters,board", [
    (31, 24, 4, None),
    (32, 40, 3, None),
    (33, 20, 3, ["Ks", "Kd", "Kh", "Kc", "2s"]),   # quads on board: large tie groups
    (34, 16, 3, ["As", "Ks", "Qs", "Js", "Ts"]),   # royal flush on board: every hand ties
    (35, 30, 3, ["2c", "2d", "7h", "7s", "9c"]),   # two pair on board
])
def test_three_way_showdowns_against_oracle(oracle, seed, nh, iters, board):
    cfg = river3(seed, nh, board)
    ours, lv = solve(cfg, iters)
    r32, _ = oracle_pair(oracle, cfg, iters, lv)
    strict(ours, r32)


@pytest.mark.gpu
def test_three_way_showdowns_fp64_at_60_hands(oracle):
    """A larger range against the FP64 restatement (the reference's own FP32
    sums drift from exact arithmetic as ranges grow)."""
    cfg = river3(36, 60)
    ours, lv = solve(cfg, 3)
    r32, r64 = oracle_pair(oracle, cfg, 3, lv)
    strict(ours, r64)
    assert diffs(ours, r64)[0] <= diffs(r32, r64)[0] + 1e-4


@pytest.mark.gpu
def test_full_size_three_player_river_solves():
    """1081 combos per player: solved (the enumeration would need ~1e9 tuple
    visits per hand and showdown), and the FP64 exploitability of the average
    strategy falls well below that of the uniform profile (one iteration).
    With three players CFR does not promise a monotone decrease, so only the
    drop from uniform play is asserted."""
    cfg = river3(37, None)
    sg = wl.AbiSubgame(cfg)
    rc, res1 = sg.solve(1)
    assert rc == 0, wl.ssg.last_error(sg.lib)
    rc, res200 = sg.solve(200)
    assert rc == 0, wl.ssg.last_error(sg.lib)
    e1 = gpu_exploitability(sg, res1["avg_strategies"])["pct"]
    e200 = gpu_exploitability(sg, res200["avg_strategies"])["pct"]
    sg.free()
    assert np.isfinite(res200["avg_strategies"]).all()
    assert 0.0 <= e200 < 0.25 * e1, (e1, e200)
