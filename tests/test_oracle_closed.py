"""Pin the oracle's closed-form FP64 checker (orc_solve_f64_closed) to its
odometer restatement of street_solve.cu.

The closed form evaluates folds and leaves with one or two counted opponents
by inclusion-exclusion over shared cards (O(H * 52) per traverser hand)
instead of enumerating opponent tuples (O(H^k)), so that the 3-player turn
at its full size (1128 hands) can be checked.  On every size where the
odometer still runs it must give the same FP64 solve: same sums, different
order, so the outputs agree to rounding (1e-10 here), and the exact zeros
(traverser hands with no compatible positive-reach tuple) stay exact.
"""
import numpy as np
import pytest

import workloads as wl

CASES = [
    # name, seed, hands/player, iterations, overrides
    ("turn3", 3, 16, 3, {}),
    ("turn3", 4, 24, 2, {}),
    ("turn3", 5, 12, 4, {"bet_sizes": [0.75], "max_raises": 1}),
    ("hu_river", 5, 60, 5, {}),
    ("river6", 5, 10, 3, {"num_players": 3, "bet_sizes": [1.0], "max_raises": 1}),
]

# One iteration only: on this small 3-player river a hand's check (three-way
# showdown, summed per tuple) and bet (everyone folds: payoff x mass) are worth
# the same; the odometer's two sums happen to round to the same double, the
# closed form's to values 1e-17 apart.  The regret is then exactly 0 in one
# and +-7e-18 in the other, which regret matching turns into a uniform versus
# a pure strategy from the next iteration on.  Any two summation orders can
# split this way (the reference's FP32 and FP64 runs too); the sums
# themselves agree to rounding.
ONE_ITERATION = [("river6", 6, 10, {"num_players": 3, "bet_sizes": [1.0], "max_raises": 1})]


def run(oracle, cfg, iters, precision):
    tree = oracle.build_tree(cfg["board"], cfg["pot"], cfg["stack"], cfg["bet_sizes"],
                             cfg["num_players"], max_raises=cfg["max_raises"])
    H, W, n = wl.padded(cfg)
    lv = wl.leaf_values_for(cfg, tree.num_leaves)
    return oracle.solve(tree, H, W, n, iters, leaf_values=lv, precision=precision, want_state=True)


@pytest.mark.parametrize("name,seed,nh,iters,over", CASES)
def test_closed_form_matches_odometer(oracle, name, seed, nh, iters, over):
    cfg = wl.config(name, seed=seed, num_hands=nh, **over)
    a = run(oracle, cfg, iters, "f64")
    b = run(oracle, cfg, iters, "f64_closed")
    assert np.array_equal(a["avg_node_ids"], b["avg_node_ids"])
    assert np.abs(a["avg_strategies"] - b["avg_strategies"]).max() <= 1e-10
    scale = max(np.abs(a["root_ev"]).max(), 1e-30)
    assert np.abs(a["root_ev"] - b["root_ev"]).max() / scale <= 1e-10
    rscale = max(np.abs(a["regrets"]).max(), 1e-30)
    assert np.abs(a["regrets"] - b["regrets"]).max() / rscale <= 1e-10
    # exact zeros stay exact: a regret row that is exactly 0 in one is in the other
    assert np.array_equal(a["regrets"] == 0, b["regrets"] == 0)


@pytest.mark.parametrize("name,seed,nh,over", ONE_ITERATION)
def test_closed_form_one_iteration(oracle, name, seed, nh, over):
    cfg = wl.config(name, seed=seed, num_hands=nh, **over)
    a = run(oracle, cfg, 1, "f64")
    b = run(oracle, cfg, 1, "f64_closed")
    rscale = max(np.abs(a["regrets"]).max(), 1e-30)
    assert np.abs(a["regrets"] - b["regrets"]).max() / rscale <= 1e-12
    assert np.abs(a["strategy_sum"] - b["strategy_sum"]).max() <= 1e-12


def test_closed_form_exact_zeros_on_blocked_hands(oracle):
    """Opponent ranges with most weights zero: many traverser hands meet no
    positive-reach tuple, where the odometer's sum is exactly 0 and the closed
    form must give exactly 0 too (not rounding residue)."""
    cfg = wl.config("turn3", seed=17, num_hands=14)
    rng = np.random.default_rng(17)
    for p in range(1, cfg["num_players"]):
        w = cfg["weights"][p].copy()
        w[rng.random(w.shape[0]) < 0.8] = 0.0
        cfg["weights"][p] = w
    a = run(oracle, cfg, 3, "f64")
    b = run(oracle, cfg, 3, "f64_closed")
    assert np.array_equal(a["regrets"] == 0, b["regrets"] == 0)
    rscale = max(np.abs(a["regrets"]).max(), 1e-30)
    assert np.abs(a["regrets"] - b["regrets"]).max() / rscale <= 1e-10
