"""The multi-street solver (fs_solve_gpu, fs_solve_gpu_extract_all) against
the reference's own sm_100a build of src/cuda/flop_solve.cu on the same
tree, hands and weights.

fs_solve_gpu returns the last iterate's root strategy; the extraction adds
the normalised average strategy of every decision node and the last
traverser's values at every node.  The two solvers sum in different orders
(the reference averages each chance node's children, this solver folds the
1 / cards weights into frontier rows), so results agree to FP32 rounding:
strategies within 1e-4, values within 1e-4 of the largest value.
"""
import ctypes
import os

import numpy as np
import pytest

import flop_solve as fsm
import street_solver_gpu as ssg
import workloads as wl

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "libref_flop_solve_gpu.so")


def ranges(seed, flop, n):
    rng = np.random.default_rng(seed)
    h, w = wl.make_ranges(rng, flop, 2, n)
    return h, w


def pair(seed, flop, n, pot, stack, sizes, iters, extract):
    if not os.path.exists(REF):
        pytest.skip("reference flop solver build not present")
    h, w = ranges(seed, flop, n)
    ours = fsm.FlopSubgame(ssg.load_library(200), flop, pot, stack, sizes, h, w)
    theirs = fsm.FlopSubgame(ctypes.CDLL(REF), flop, pot, stack, sizes, h, w)
    a = ours.solve(iters, extract=extract)
    b = theirs.solve(iters, extract=extract)
    dec = fsm.tree_arrays(ours.td)[4]
    ours.free()
    theirs.free()
    return a, b, dec


@pytest.mark.gpu
@pytest.mark.parametrize("seed,flop,n,pot,stack,sizes,iters", [
    (1, [0, 13, 26], 12, 1000, 5000, [0.75], 4),
    (2, [51, 7, 22], 20, 650, 9750, [0.5, 1.0], 3),
    (3, [3, 17, 40], 40, 400, 1200, [1.0], 6),
])
def test_root_strategy_against_reference(seed, flop, n, pot, stack, sizes, iters):
    a, b, _ = pair(seed, flop, n, pot, stack, sizes, iters, False)
    assert a["root_player"] == b["root_player"] and a["root_num_actions"] == b["root_num_actions"]
    assert np.abs(a["root_strategy"] - b["root_strategy"]).max() <= 1e-4


@pytest.mark.gpu
def test_extract_all_against_reference():
    """Every decision node's average strategy and every node's value after 5
    iterations.  On 16-hand ranges some hands' values tie exactly in one
    summation order and not in another, and regret matching turns that into a
    different strategy, so the element-wise bound is the envelope of
    tests/test_parity_gpu.py: this solver may be no further from the FP64
    restatement (oracle/fs_oracle.c) than ENVELOPE times the reference's own
    FP32 distance from it, plus the 1e-4 tolerances."""
    from oracle.oracle import FlopOracle
    from test_parity_gpu import ENVELOPE
    seed, flop, n, pot, stack, sizes, iters = 4, [9, 21, 35], 16, 1000, 5000, [0.75], 5
    a, b, dec = pair(seed, flop, n, pot, stack, sizes, iters, True)
    assert np.array_equal(a["turn_root_indices"], b["turn_root_indices"])
    assert np.array_equal(a["turn_root_cards"], b["turn_root_cards"])
    assert len(a["turn_root_indices"]) > 0 and a["max_hands"] == b["max_hands"]
    lib = fsm.bind(ssg.load_library(200))
    h, w = ranges(seed, flop, n)
    sg = fsm.FlopSubgame(lib, flop, pot, stack, sizes, h, w)
    nodes, ch, _, nd, _, _ = fsm.tree_arrays(sg.td)
    H = np.zeros((2, 200, 2), np.int32)
    W = np.zeros((2, 200), np.float32)
    for p in range(2):
        H[p, :n], W[p, :n] = h[p], w[p]
    e = FlopOracle().solve(nodes, ch, nd, sg.td.max_depth, H, W, np.array([n, n], np.int32), iters, "f64")
    sg.free()
    da = np.abs(a["all_avg_strategies"][dec] - e["all_avg_strategies"][dec]).max()
    db = np.abs(b["all_avg_strategies"][dec] - e["all_avg_strategies"][dec]).max()
    assert da <= ENVELOPE * db + 1e-4, f"avg strategy: ours-f64 {da}, reference f32-f64 {db}"
    scale = max(np.abs(e["all_cfv"]).max(), 1e-30)
    va = np.abs(a["all_cfv"] - e["all_cfv"]).max() / scale
    vb = np.abs(b["all_cfv"] - e["all_cfv"]).max() / scale
    assert va <= ENVELOPE * vb + 1e-4, f"values: ours-f64 {va}, reference f32-f64 {vb}"
