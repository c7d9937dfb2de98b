"""The multi-street solver (fs_solve_gpu, fs_solve_gpu_extract_all) on the GPU
against the reference and its restatement.

* Root strategies against the reference's own sm_100a build of
  src/cuda/flop_solve.cu (fs_solve_gpu, same tree, hands, weights and
  iterations).
* Every node's average strategy and value (extract_all) against the oracle's
  restatement (oracle/fs_oracle.c, pinned to the reference's root strategies
  by tests/test_flop_oracle.py); the reference's own extraction cannot serve:
  it overflows a 52-entry host buffer with the 245 turn roots of these trees
  (flop_solve.cu:1529-1543).

The solvers sum in different orders (the reference averages each chance
node's children, this solver folds the 1 / cards weights into frontier rows
and sums terminals in FP64 closed forms).  On these small ranges some hands'
values tie exactly in one order and not in another, which regret matching
turns into different strategies, so the bound is the envelope rule of
tests/test_parity_gpu.py: this solver may be no further from the FP64
restatement than ENVELOPE times the reference arithmetic's own distance from
it (the reference's build for root strategies, the float restatement
elsewhere), plus the 1e-4 tolerances.
"""
import ctypes
import os

import numpy as np
import pytest

import flop_solve as fsm
import street_solver_gpu as ssg
import workloads as wl
from test_parity_gpu import ENVELOPE

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "libref_flop_solve_gpu.so")


def setup(seed, flop, n, pot, stack, sizes):
    h, w = wl.make_ranges(np.random.default_rng(seed), flop, 2, n)
    sg = fsm.FlopSubgame(ssg.load_library(200), flop, pot, stack, sizes, h, w)
    H = np.zeros((2, 200, 2), np.int32)
    W = np.zeros((2, 200), np.float32)
    for p in range(2):
        H[p, :n], W[p, :n] = h[p], w[p]
    return sg, h, w, H, W


def oracle_runs(sg, H, W, n, iters):
    from oracle.oracle import FlopOracle
    nodes, ch, _, nd, dec, _ = fsm.tree_arrays(sg.td)
    o = FlopOracle()
    nh = np.array([n, n], np.int32)
    r32 = o.solve(nodes, ch, nd, sg.td.max_depth, H, W, nh, iters, "f32")
    r64 = o.solve(nodes, ch, nd, sg.td.max_depth, H, W, nh, iters, "f64")
    return r32, r64, dec


@pytest.mark.gpu
@pytest.mark.parametrize("seed,flop,n,pot,stack,sizes,iters", [
    (1, [0, 13, 26], 12, 1000, 5000, [0.75], 4),
    (2, [51, 7, 22], 20, 650, 9750, [0.5, 1.0], 3),
    (3, [3, 17, 40], 40, 400, 1200, [1.0], 6),
])
def test_root_strategy_against_reference(seed, flop, n, pot, stack, sizes, iters):
    if not os.path.exists(REF):
        pytest.skip("reference flop solver build not present")
    sg, h, w, H, W = setup(seed, flop, n, pot, stack, sizes)
    ours = sg.solve(iters)
    theirs = fsm.FlopSubgame(ctypes.CDLL(REF), flop, pot, stack, sizes, h, w)
    ref = theirs.solve(iters)
    theirs.free()
    _, r64, _ = oracle_runs(sg, H, W, n, iters)
    sg.free()
    assert ours["root_player"] == ref["root_player"] and ours["root_num_actions"] == ref["root_num_actions"]
    da = np.abs(ours["root_strategy"] - r64["root_strategy"]).max()
    db = np.abs(ref["root_strategy"] - r64["root_strategy"]).max()
    print(f"root strategy: ours-f64 {da:.2e}, reference-f64 {db:.2e}, ours-reference "
          f"{np.abs(ours['root_strategy'] - ref['root_strategy']).max():.2e}")
    assert da <= ENVELOPE * db + 1e-4


@pytest.mark.gpu
@pytest.mark.parametrize("iters", [1, 5])
def test_extract_all_against_restatement(iters):
    seed, flop, n, pot, stack, sizes = 4, [9, 21, 35], 16, 1000, 5000, [0.75]
    sg, h, w, H, W = setup(seed, flop, n, pot, stack, sizes)
    a = sg.solve(iters, extract=True)
    r32, r64, dec = oracle_runs(sg, H, W, n, iters)
    nodes = fsm.tree_arrays(sg.td)[0]
    sg.free()
    # turn roots: the decision children of the flop-ending chance nodes, by node id
    chance3 = [x for x in range(nodes.shape[0]) if nodes[x, 0] == 3 and nodes[x, 12] == 3]
    assert len(a["turn_root_indices"]) == 49 * len(chance3)
    assert np.all(nodes[a["turn_root_indices"], 12] == 4)
    assert np.array_equal(nodes[a["turn_root_indices"], 10], a["turn_root_cards"])
    da = np.abs(a["all_avg_strategies"][dec] - r64["all_avg_strategies"][dec]).max()
    db = np.abs(r32["all_avg_strategies"][dec] - r64["all_avg_strategies"][dec]).max()
    scale = max(np.abs(r64["all_cfv"]).max(), 1e-30)
    va = np.abs(a["all_cfv"] - r64["all_cfv"]).max() / scale
    vb = np.abs(r32["all_cfv"] - r64["all_cfv"]).max() / scale
    print(f"{iters} iterations: avg strategy ours-f64 {da:.2e} f32-f64 {db:.2e}; values ours-f64 {va:.2e} "
          f"f32-f64 {vb:.2e}")
    assert da <= ENVELOPE * db + 1e-4, f"avg strategy: ours-f64 {da}, f32-f64 {db}"
    assert va <= ENVELOPE * vb + 1e-4, f"values: ours-f64 {va}, f32-f64 {vb}"
