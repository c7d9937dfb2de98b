"""GPU parity at the benchmark sizes.

* The 3-player turn with continuation leaves at its full size (1128 combos
  per player, 21,436 nodes, 15,616 leaf terminals): the odometer is out of
  reach there (O(H^3) per two-opponent terminal), so the checker is the
  oracle's closed-form FP64 solve (orc_solve_f64_closed), itself pinned to
  the odometer on every size where that runs (tests/test_oracle_closed.py).
  Element-wise after 1 and 3 iterations: average strategies within 1e-4
  absolute, root values within 1e-4 relative, root strategy within 1e-4.
* The heads-up river at its full size (1081 combos each) for the full 1000
  iterations against the oracle's FP32 (reference arithmetic and order) and
  FP64 solves, under the envelope rule of tests/test_parity_gpu.py: CFR
  amplifies rounding over 1000 iterations, so the solver may not be further
  from FP64 than ENVELOPE times the reference arithmetic's own distance from
  it (plus the 1e-4 tolerances).
"""
import numpy as np
import pytest

import workloads as wl
from test_parity_gpu import ENVELOPE, EV_RTOL, STRAT_ATOL, check_layout, diffs, envelope, solve


def oracle_solve(oracle, cfg, iters, lv, precision):
    tree = oracle.build_tree(cfg["board"], cfg["pot"], cfg["stack"], cfg["bet_sizes"],
                             cfg["num_players"], max_raises=cfg["max_raises"])
    H, W, nh = wl.padded(cfg)
    return oracle.solve(tree, H, W, nh, iters, leaf_values=lv, precision=precision)


@pytest.mark.gpu
@pytest.mark.parametrize("iters", [1, 3])
def test_turn3_full_size_against_closed_form_oracle(oracle, iters):
    cfg = wl.config("turn3", seed=0)
    assert all(len(h) == 1128 for h in cfg["hands"])
    ours, lv = solve(cfg, iters)
    ref = oracle_solve(oracle, cfg, iters, lv, "f64_closed")
    check_layout(ours, ref)
    assert ours["avg_strategies"].shape[0] > 5000   # every decision node of the full tree
    ds, de, dr = diffs(ours, ref)
    assert ds <= STRAT_ATOL, f"avg strategy diff {ds}"
    assert de <= EV_RTOL, f"root value rel diff {de}"
    assert dr <= STRAT_ATOL, f"root strategy diff {dr}"


@pytest.mark.gpu
def test_hu_river_full_size_1000_iterations(oracle):
    cfg = wl.config("hu_river", seed=0)
    assert cfg["iterations"] == 1000 and all(len(h) == 1081 for h in cfg["hands"])
    ours, lv = solve(cfg, 1000)
    r32 = oracle_solve(oracle, cfg, 1000, lv, "f32")
    r64 = oracle_solve(oracle, cfg, 1000, lv, "f64")
    envelope(ours, r32, r64)
    ds, de, _ = diffs(ours, r64)
    rs, re, _ = diffs(r32, r64)
    print(f"1000 iterations: ours-f64 strategy {ds:.2e} value {de:.2e}; "
          f"reference f32-f64 strategy {rs:.2e} value {re:.2e} (envelope x{ENVELOPE})")
