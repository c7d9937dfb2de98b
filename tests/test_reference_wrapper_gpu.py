"""The drop-in, shown with the reference's own consumer of the C ABI.

python/street_solver_gpu.py and python/solver.py of the reference, copied
unmodified into oracle/_ref/wrapper/python/ by oracle/build_ref.py, are placed
in a temporary tree whose build/street_solve.so (the path the module loads,
street_solver_gpu.py:48-57) is a link to this repository's
libstreet_solve.so (200-hand layout).  The module then runs exactly as in
the reference: StreetSolverGPU builds the tree, fills ranges and leaf values,
solve() calls ss_solve_gpu, the read-outs (get_strategy with and without
frozen actions, get_avg_strategy) walk the returned SSOutput, and free()
calls ss_free_tree / ss_free_output (the reference library would also free
the module's own leaf-value array there; this one leaves caller memory
alone, so the module's later garbage collection is safe).

Results are compared with the oracle (the C restatement of street_solve.cu)
on the same tree, hands, weights, leaf values and frozen actions.
"""
import ctypes
import gc
import importlib.util
import os
import shutil
import sys

import numpy as np
import pytest

import workloads as wl
from test_parity_gpu import STRAT_ATOL, EV_RTOL

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
WRAPPER = os.path.join(ROOT, "oracle", "_ref", "wrapper", "python")
LIB = os.path.join(ROOT, "poker-solver_b200", "lib", "libstreet_solve.so")


@pytest.fixture(scope="module")
def refmod(tmp_path_factory):
    if not os.path.exists(os.path.join(WRAPPER, "street_solver_gpu.py")):
        pytest.skip("reference wrapper not copied (oracle/build_ref.py needs the reference sources)")
    base = tmp_path_factory.mktemp("ref_tree")
    os.makedirs(base / "python")
    os.makedirs(base / "build")
    for name in ("street_solver_gpu.py", "solver.py"):
        shutil.copyfile(os.path.join(WRAPPER, name), base / "python" / name)
    os.symlink(LIB, base / "build" / "street_solve.so")
    sys.path.insert(0, str(base / "python"))
    try:
        spec = importlib.util.spec_from_file_location("ref_street_solver_gpu",
                                                      base / "python" / "street_solver_gpu.py")
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        yield mod
    finally:
        sys.path.remove(str(base / "python"))


def out_arrays(solver):
    """The SSOutput the module holds, as numpy arrays (reference layout)."""
    o = solver._output
    mh = o.max_hands
    avg = np.ctypeslib.as_array(o.avg_strategies, shape=(o.num_avg_nodes * 8 * mh,)).copy()
    ids = np.ctypeslib.as_array(o.avg_strategy_node_ids, shape=(o.num_avg_nodes,)).copy()
    ev = np.ctypeslib.as_array(o.root_ev, shape=(mh,)).copy()
    return avg.reshape(o.num_avg_nodes, 8, mh), ids, ev


def oracle_for(oracle, solver, iters, lv=None, frozen=None):
    t = solver._tree
    np_ = solver.num_players
    tree = oracle.build_tree(solver.board_cards, t.starting_pot, t.effective_stack, solver.bet_sizes,
                             np_, max_raises=3)
    mh = max(len(h) for h in solver.player_hands)
    H = np.zeros((np_, mh, 2), np.int32)
    W = np.zeros((np_, mh), np.float32)
    for p, hands in enumerate(solver.player_hands):
        for i, (c0, c1, w) in enumerate(hands):
            H[p, i] = (c0, c1)
            W[p, i] = w
    nh = np.array([len(h) for h in solver.player_hands], np.int32)
    return tree, oracle.solve(tree, H, W, nh, iters, leaf_values=lv, frozen=frozen)


def ranges(cfg):
    return [[(int(a), int(b), float(w)) for (a, b), w in zip(h, ws)]
            for h, ws in zip(cfg["hands"], cfg["weights"])]


def compare(solver, ref):
    avg, ids, ev = out_arrays(solver)
    assert np.array_equal(ids, ref["avg_node_ids"])
    assert np.abs(avg - ref["avg_strategies"]).max() <= STRAT_ATOL
    scale = max(np.abs(ref["root_ev"]).max(), 1e-30)
    assert np.abs(ev - ref["root_ev"]).max() / scale <= EV_RTOL


@pytest.mark.gpu
def test_reference_module_river(refmod, oracle):
    cfg = wl.config("hu_river", seed=31, num_hands=150)
    solver = refmod.StreetSolverGPU(board=cfg["board"], pot_bb=1.0, stack_bb=4.0,
                                    player_ranges=ranges(cfg), bet_sizes=[0.5, 1.0])
    assert os.path.realpath(refmod._LIB._name) == os.path.realpath(LIB)
    solver.solve(iterations=6)
    tree, ref = oracle_for(oracle, solver, 6)
    compare(solver, ref)
    # read-outs of the module against the oracle's arrays
    labels = refmod._build_labels_at_node(solver._tree, 0)
    na = ref["root_num_actions"]
    for h in (0, 17, 149):
        got = solver.get_strategy(0, hand_idx=h)
        want = {labels[a]: float(ref["root_strategy"][a, h]) for a in range(na)
                if ref["root_strategy"][a, h] > 0.001}
        assert set(got) == set(want)
        assert all(abs(got[k] - want[k]) <= STRAT_ATOL for k in want)
    avg = solver.get_avg_strategy(1)
    di = int(np.nonzero(tree.col("player")[ref["avg_node_ids"]] == 1)[0][0])
    node = int(ref["avg_node_ids"][di])
    lab1 = refmod._build_labels_at_node(solver._tree, node)
    for h, (c0, c1, _) in enumerate(solver.player_hands[1][:40]):
        got = avg[(min(c0, c1), max(c0, c1))]
        for a, lbl in enumerate(lab1):
            f = float(ref["avg_strategies"][di, a, h])
            if f > 0.001 + STRAT_ATOL:
                assert abs(got[lbl] - f) <= STRAT_ATOL
    solver.free()
    solver.free()       # idempotent, as in the reference module


@pytest.mark.gpu
def test_reference_module_turn_leaves_and_frozen(refmod, oracle):
    cfg = wl.config("turn3", seed=32, num_hands=14, bet_sizes=[0.75], max_raises=1)
    rng = np.random.default_rng(32)
    made = {}

    def leaf_fn(tree, player_hands, max_h, pot):
        lv = rng.normal(0.0, 40.0, (tree.num_leaves, len(player_hands), max_h)).astype(np.float32)
        made["lv"] = lv
        return lv

    solver = refmod.StreetSolverGPU(board=cfg["board"], pot_bb=1.5, stack_bb=5.0,
                                    player_ranges=ranges(cfg), bet_sizes=[0.75],
                                    leaf_value_fn=leaf_fn)
    assert solver._tree.num_leaves > 0 and "lv" in made
    # freeze player 0's first action (the module's own A3 walk)
    first = refmod._build_labels_at_node(solver._tree, 0)[1]
    solver.set_frozen_actions([first], hero_player=0)
    n = solver._tree.num_nodes
    frozen = np.ctypeslib.as_array(solver._tree.frozen_action, shape=(n,)).copy()
    assert frozen[0] == 1
    solver.solve(iterations=5)
    tree, ref = oracle_for(oracle, solver, 5, lv=made["lv"], frozen=frozen)
    compare(solver, ref)
    got = solver.get_strategy(0, hand_idx=3)
    assert got == {first: 1.0}
    # the walk through frozen actions reaches player 1's node below it
    nxt = solver.get_strategy(1, hand_idx=2, frozen_actions=[first])
    assert abs(sum(nxt.values()) - 1.0) <= 0.01
    solver.free()
    del solver
    gc.collect()
