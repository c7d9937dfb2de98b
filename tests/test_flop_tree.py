"""The multi-street tree builder (fs_build_tree) against the reference's own
(src/cuda/flop_solve.cu built by oracle/build_ref.py; its builder is host
code, so it runs here): every node field, the children array, BFS order,
depths and index lists equal, for several flops, pots, stacks and bet sets.
Also the ABI sizes of the mirrors and the builder's argument checks."""
import ctypes
import os

import numpy as np
import pytest

import flop_solve as fsm
import street_solver_gpu as ssg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "libref_flop_solve_gpu.so")

CASES = [
    # flop, pot, stack, bet sizes
    ([0, 13, 26], 1000, 5000, [0.75]),
    ([51, 7, 22], 650, 9750, [0.5, 1.0]),
    ([3, 4, 5], 100, 400, [0.33, 0.75, 1.5]),
    ([10, 20, 30], 400, 300, [0.5]),          # short stack: all-ins capped on the flop
    ([8, 9, 44], 2000, 9000, [1.0, 2.0]),     # turn / river stacks reach 0 below big flop bets
]


def build(lib, flop, pot, stack, sizes):
    fsm.bind(lib)
    td = fsm.FSTreeData()
    b = (ctypes.c_int * 3)(*flop)
    s = (ctypes.c_float * len(sizes))(*sizes)
    rc = lib.fs_build_tree(b, pot, stack, s, len(sizes), ctypes.byref(td))
    assert rc == 0
    arrs = fsm.tree_arrays(td)
    meta = (td.num_nodes, td.num_children_total, td.max_depth, td.num_decision_nodes, td.num_showdown_nodes)
    lib.fs_free_tree(ctypes.byref(td))
    return arrs, meta


def test_layout_sizes():
    assert ctypes.sizeof(fsm.FSNode) == 52
    assert ctypes.sizeof(fsm.FSTreeData) == 8 + 8 + 4 + 4 + 2 * 200 * 2 * 4 + 2 * 200 * 4 + 8 + 8 + 8 + 4 + 4 + 8 + 4 + 4 + 8 + 4 + 4


@pytest.mark.skipif(not os.path.exists(REF), reason="reference flop solver build not present")
@pytest.mark.parametrize("flop,pot,stack,sizes", CASES)
def test_tree_equals_reference(flop, pot, stack, sizes):
    ours = ssg.load_library(200)
    theirs = ctypes.CDLL(REF)
    a, ma = build(ours, flop, pot, stack, sizes)
    b, mb = build(theirs, flop, pot, stack, sizes)
    assert ma == mb
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_tree_shape():
    lib = ssg.load_library(200)
    (nodes, ch, lo, nd, dec, sd), meta = build(lib, [0, 13, 26], 1000, 5000, [0.75])
    types = nodes[:, 0]
    assert set(np.unique(types)) <= {0, 1, 2, 3}
    # every chance node deals every undealt card; showdowns hold five cards
    for x in np.nonzero(types == 3)[0]:
        assert nodes[x, 2] == 52 - nodes[x, 12]
    assert np.all(nodes[types == 2, 12] == 5)
    assert lo[0] == 0 and len(np.unique(lo)) == len(lo)


def test_bad_arguments():
    lib = fsm.bind(ssg.load_library(200))
    td = fsm.FSTreeData()
    s = (ctypes.c_float * 1)(0.75)
    assert lib.fs_build_tree((ctypes.c_int * 3)(1, 1, 2), 100, 400, s, 1, ctypes.byref(td)) != 0
    assert lib.fs_build_tree((ctypes.c_int * 3)(1, 2, 60), 100, 400, s, 1, ctypes.byref(td)) != 0
    assert not td.nodes
