"""Pin the multi-street oracle (oracle/fs_oracle.c) to the reference: its
float solve reproduces the reference's own GPU results
(tests/golden/flop_ref_*.npz, made by make_flop_golden.py with the
reference's sm_100a build) -- root strategy, normalised average strategies
and values at the sampled nodes.  The float restatement repeats the
reference's operations in its order, fused multiply-adds included, so the
bound is 1e-6 (strategies) and 1e-6 of the largest value.  The double solve
follows the same algorithm; where two hands' values tie exactly in one
precision and not the other, regret matching turns the difference into a
different strategy, so only its root strategy is held (within 1e-4) on
these small ranges."""
import ctypes
import glob
import os

import numpy as np
import pytest

import flop_solve as fsm
import street_solver_gpu as ssg

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FIXTURES = sorted(glob.glob(os.path.join(GOLDEN, "flop_ref_*.npz")))


def tree_of(g):
    lib = fsm.bind(ssg.load_library(200))
    td = fsm.FSTreeData()
    flop = [int(c) for c in g["flop"]]
    sizes = [float(x) for x in g["bet_sizes"]]
    rc = lib.fs_build_tree((ctypes.c_int * 3)(*flop), int(g["pot"]), int(g["stack"]),
                           (ctypes.c_float * len(sizes))(*sizes), len(sizes), ctypes.byref(td))
    assert rc == 0 and td.num_nodes == int(g["num_nodes"])
    nodes, ch, _, nd, _, _ = fsm.tree_arrays(td)
    max_depth = td.max_depth
    lib.fs_free_tree(ctypes.byref(td))
    return nodes, ch, nd, max_depth


def inputs(g):
    H = np.zeros((2, 200, 2), np.int32)
    W = np.zeros((2, 200), np.float32)
    nh = np.array([len(g["hands"][0]), len(g["hands"][1])], np.int32)
    for p in range(2):
        H[p, :nh[p]] = g["hands"][p]
        W[p, :nh[p]] = g["weights"][p]
    return H, W, nh


@pytest.mark.skipif(not FIXTURES, reason="no reference flop fixtures")
@pytest.mark.parametrize("path", FIXTURES, ids=lambda p: os.path.basename(p)[9:-4])
def test_oracle_matches_reference_gpu(oracle_flop, path):
    g = np.load(path)
    nodes, ch, nd, md = tree_of(g)
    H, W, nh = inputs(g)
    ids = g["node_ids"]
    r = oracle_flop.solve(nodes, ch, nd, md, H, W, nh, int(g["iterations"]), "f32")
    assert np.abs(r["root_strategy"] - g["root_strategy"]).max() <= 1e-6
    assert np.abs(r["all_avg_strategies"][ids] - g["avg"]).max() <= 1e-6
    scale = max(np.abs(g["cfv"]).max(), 1e-30)
    assert np.abs(r["all_cfv"][ids] - g["cfv"]).max() / scale <= 1e-6
    r64 = oracle_flop.solve(nodes, ch, nd, md, H, W, nh, int(g["iterations"]), "f64")
    assert np.abs(r64["root_strategy"] - g["root_strategy"]).max() <= 1e-4


@pytest.fixture(scope="module")
def oracle_flop():
    from oracle.oracle import FlopOracle
    return FlopOracle()
