"""Pin the multi-street oracle (oracle/fs_oracle.c) to the reference: its
float solve reproduces the root strategy of the reference's own GPU solve
(tests/golden/flop_ref_*.npz, made by make_flop_golden.py with the
reference's sm_100a build) after 1, 2, 3 and 5 iterations.  The float
restatement repeats the reference's operations in its order, fused
multiply-adds included, so the bound is 1e-6.  (The reference's extraction
entry point overflows a host buffer on every full tree, so the root strategy
is what the reference itself can give.)  The double solve must stay within
1e-4 of it at the root after one iteration."""
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
    ks = [int(k) for k in g["iterations"]]
    r = oracle_flop.solve(nodes, ch, nd, md, H, W, nh, max(ks), "f32", snapshots=ks, full=False)
    for k in ks:
        want = g[f"root_strategy_{k}"]
        assert np.abs(r["root_snapshots"][k] - want).max() <= 1e-6, f"{k} iterations"
    # the double solve after one iteration (later ones drift apart through
    # regret-matching ties, which float rounding breaks differently)
    r64 = oracle_flop.solve(nodes, ch, nd, md, H, W, nh, 1, "f64", full=False)
    assert np.abs(r64["root_strategy"] - g["root_strategy_1"]).max() <= 1e-4


@pytest.fixture(scope="module")
def oracle_flop():
    from oracle.oracle import FlopOracle
    return FlopOracle()
