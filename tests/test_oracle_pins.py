"""Pin the oracle: its C restatement of street_solve.cu and of hand_eval.h
must reproduce the reference bit for bit.

* golden fixtures (tests/golden/, made by make_golden.py from the reference
  itself): trees and solve outputs of small seeded cases, an all-hands
  checksum of the reference evaluator and a random sample of strengths;
* the reference builds in oracle/_ref/ when present (same container, or the
  GPU box, which receives them prebuilt).
"""
import ctypes
import glob
import json
import os

import numpy as np
import pytest

from oracle.oracle import RefHandEval, RefStreetSolve, ref_available

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
SOLVE_FIXTURES = sorted(glob.glob(os.path.join(GOLDEN, "ref_solve_*.npz")))


def fixture_tree(oracle, g):
    return oracle.build_tree([int(c) for c in g["board"]], int(g["pot"]), int(g["stack"]),
                             [float(x) for x in g["bet_sizes"]], int(g["num_players"]),
                             max_raises=int(g["max_raises"]))


@pytest.mark.parametrize("path", SOLVE_FIXTURES, ids=lambda p: os.path.basename(p)[10:-4])
def test_oracle_matches_reference_fixture(oracle, path):
    g = np.load(path)
    tree = fixture_tree(oracle, g)
    assert np.array_equal(tree.nodes, g["nodes"])
    assert np.array_equal(tree.children, g["children"])
    assert np.array_equal(tree.level_order, g["level_order"])
    assert np.array_equal(tree.node_depth, g["node_depth"])
    assert tree.max_depth == int(g["max_depth"]) and tree.num_leaves == int(g["num_leaves"])
    lv = g["leaf_values"] if g["leaf_values"].size else None
    fz = g["frozen"] if g["frozen"].size else None
    out = oracle.solve(tree, g["hands"], g["weights"], g["num_hands"], int(g["iterations"]),
                       leaf_values=lv, frozen=fz)
    for k in ("root_strategy", "root_ev", "avg_strategies", "avg_node_ids"):
        assert np.array_equal(out[k], g[k]), k
    assert out["root_player"] == int(g["root_player"])


def test_oracle_evaluator_sample(oracle):
    g = np.load(os.path.join(GOLDEN, "hand_rank_sample.npz"))
    out = np.zeros(g["cards"].shape[0], np.uint32)
    oracle.lib.orc_eval7_many(g["cards"].ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                              ctypes.c_long(len(out)),
                              out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)))
    assert np.array_equal(out, g["strength"])


def test_oracle_evaluator_all_hands(oracle):
    ref = json.load(open(os.path.join(GOLDEN, "hand_rank_all.json")))
    oracle.lib.orc_eval7_checksum.restype = ctypes.c_uint64
    hist = (ctypes.c_uint64 * 10)()
    chk = oracle.lib.orc_eval7_checksum(hist)
    assert f"{chk:#018x}" == ref["checksum"]
    assert list(hist) == ref["category_counts"]
    assert sum(hist) == 133784560


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(GOLDEN), "..", "oracle", "_ref",
                                                    "libref_handeval.so")),
                    reason="reference evaluator build not present")
def test_reference_evaluator_sample_live(oracle):
    rng = np.random.default_rng(3)
    cards = np.array([rng.choice(52, 7, replace=False) for _ in range(5000)], np.int32)
    ref = RefHandEval().eval7_many(cards)
    out = np.zeros(len(cards), np.uint32)
    oracle.lib.orc_eval7_many(cards.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), ctypes.c_long(len(out)),
                              out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)))
    assert np.array_equal(out, ref)


LIVE_CASES = [
    # board size, players, hands, iterations, raise cap, bet sizes
    (5, 2, 25, 15, 2, [0.5, 1.0]),
    (5, 2, 18, 10, 3, [0.33, 0.75, 1.5]),
    (4, 2, 14, 6, 3, [0.5, 1.0]),
    (3, 2, 10, 3, 2, [0.75]),
    (5, 3, 7, 3, 2, [1.0]),
    (4, 3, 6, 2, 3, [0.75]),
    (5, 4, 5, 2, 2, [1.0]),
]


@pytest.mark.parametrize("nb,np_,nh,iters,raises,sizes", LIVE_CASES)
def test_oracle_matches_reference_live(oracle, nb, np_, nh, iters, raises, sizes):
    if not ref_available(200, raises):
        pytest.skip("reference CPU build not present")
    import workloads as wl
    rng = np.random.default_rng(1000 + nb * 10 + np_)
    board = [int(c) for c in rng.permutation(52)[:nb]]
    cfg = {"board": board, "pot": 120, "stack": 480, "bet_sizes": sizes, "max_raises": raises,
           "num_players": np_, "seed": 5, "leaf_sigma": 30.0}
    cfg["hands"], cfg["weights"] = wl.make_ranges(rng, board, np_, nh, zero_frac=0.2)
    ref = RefStreetSolve(200, raises, "cpu")
    td = ref.build(board, 120, 480, sizes, np_)
    rt = ref.tree(td)
    tree = oracle.build_tree(board, 120, 480, sizes, np_, max_raises=raises)
    assert np.array_equal(rt.nodes, tree.nodes) and np.array_equal(rt.children, tree.children)
    H, W, n = wl.padded(cfg)
    lv = wl.leaf_values_for(cfg, td.num_leaves)
    r = ref.solve(td, H, W, n, iters, leaf_values=lv)
    ref.free(td)
    o = oracle.solve(tree, H, W, n, iters, leaf_values=lv)
    for k in ("root_strategy", "root_ev", "avg_strategies", "avg_node_ids"):
        assert np.array_equal(r[k], o[k]), k


def test_exploitability_oracle_basics(oracle):
    """NashConv is >= 0, and a solved heads-up river is far less exploitable
    than the uniform profile."""
    import workloads as wl
    cfg = wl.config("hu_river", seed=4, num_hands=20)
    tree = oracle.build_tree(cfg["board"], cfg["pot"], cfg["stack"], cfg["bet_sizes"], 2,
                             max_raises=cfg["max_raises"])
    H, W, n = wl.padded(cfg)
    ndec = len(tree.decision_nodes())
    na = tree.col("num_children")[tree.decision_nodes()]
    uni = np.zeros((ndec, 8, H.shape[1]), np.float32)
    for i, a in enumerate(na):
        uni[i, :a, :] = 1.0 / a
    e_uni = oracle.exploitability(tree, H, W, n, uni)
    out = oracle.solve(tree, H, W, n, 300)
    e_cfr = oracle.exploitability(tree, H, W, n, out["avg_strategies"])
    assert e_uni["nashconv"] >= 0 and e_cfr["nashconv"] >= -1e-9
    assert e_cfr["exploitability_pct"] < 0.25 * e_uni["exploitability_pct"]
