"""CPU checks of the product library: it loads, exports every symbol of
include/street_solve.h, keeps the reference struct layouts, builds exactly
the reference trees (node ids, children, leaf numbering, BFS order), rejects
malformed input with an error code and a message, and has no CPU fallback."""
import ctypes
import os
import re

import numpy as np
import pytest

import street_solver_gpu as ssg
import workloads as wl
from conftest import HAVE_GPU, ROOT

HEADER = os.path.join(ROOT, "include", "street_solve.h")


def header_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ss_[a-z0-9_]+)\s*\(", text)))


@pytest.mark.parametrize("max_hands", [200, 1326])
def test_library_loads_and_exports_every_symbol(max_hands):
    lib = ssg.load_library(max_hands)
    names = header_functions()
    assert "ss_build_tree" in names and "ss_solve_gpu" in names
    for name in names:
        assert hasattr(lib, name), f"{name} not exported"


@pytest.mark.parametrize("max_hands", [200, 1326])
def test_abi_layout(max_hands):
    lib = ssg.load_library(max_hands)
    info = ssg.SSAbiInfo()
    assert lib.ss_abi_info(ctypes.byref(info)) == 0
    assert info.max_hands == max_hands
    assert info.sizeof_node == ctypes.sizeof(ssg.SSNode) == 104
    assert info.sizeof_tree == ctypes.sizeof(ssg.tree_struct(max_hands))
    assert info.sizeof_output == ctypes.sizeof(ssg.SSOutput)
    # the reference layout with 200 hands (street_solve.cuh:69-122)
    if max_hands == 200:
        T = ssg.tree_struct(200)
        assert T.hands.offset == 28 and T.weights.offset == 28 + 6 * 200 * 8


TREE_CASES = [
    # board size, players, bet sizes, raise cap, acting order
    (5, 2, [0.5, 1.0], 2, None),
    (5, 2, [0.33, 0.75, 1.5], 3, None),
    (5, 2, [0.5, 1.0], 2, [1, 0]),
    (4, 2, [0.33, 0.75, 1.5], 3, None),
    (3, 2, [0.5], 1, None),
    (5, 3, [0.5, 1.0], 2, None),
    (4, 3, [0.33, 0.75, 1.5], 3, None),
    (4, 3, [0.75], 2, [2, 0, 1]),
    (5, 4, [0.5, 1.0], 2, None),
    (4, 4, [1.0], 1, None),
    (5, 5, [1.0], 2, None),
    (5, 6, [0.5, 1.0], 2, None),
    (5, 2, [], 2, None),
    (5, 2, [0.2, 0.4, 0.6, 0.8], 3, None),
]


@pytest.mark.parametrize("nb,np_,sizes,raises,order", TREE_CASES)
def test_tree_matches_oracle(oracle, nb, np_, sizes, raises, order):
    rng = np.random.default_rng(nb * 100 + np_)
    board = [int(c) for c in rng.permutation(52)[:nb]]
    cfg = {"board": board, "pot": 300, "stack": 1000, "bet_sizes": sizes, "max_raises": raises,
           "num_players": np_, "seed": 1}
    cfg["hands"], cfg["weights"] = wl.make_ranges(rng, board, np_, 5)
    sg = wl.AbiSubgame(cfg, acting_order=order)
    nodes, ch, lo, nd = sg.tree_arrays()
    t = oracle.build_tree(board, 300, 1000, sizes, np_, acting_order=order, max_raises=raises)
    assert np.array_equal(nodes, t.nodes)
    assert np.array_equal(ch, t.children)
    assert np.array_equal(lo, t.level_order)
    assert np.array_equal(nd, t.node_depth)
    assert sg.td.max_depth == t.max_depth and sg.td.num_leaves == t.num_leaves
    types = nodes[:, 0]
    for name, code, cnt in (("decision", 0, sg.td.num_decision_nodes), ("fold", 1, sg.td.num_fold_nodes),
                            ("showdown", 2, sg.td.num_showdown_nodes), ("leaf", 4, sg.td.num_leaf_nodes)):
        assert int((types == code).sum()) == cnt, name
    sg.free()


def test_benchmark_tree_sizes():
    """Node counts of the three benchmark shapes (the reference builder
    gives 51 / 21,436 / 19,579)."""
    for name, n in (("hu_river", 51), ("turn3", 21436), ("river6", 19579)):
        sg = wl.AbiSubgame(wl.config(name, seed=0, num_hands=4))
        assert sg.td.num_nodes == n
        sg.free()


def test_default_raise_cap_is_reference():
    cfg = wl.config("hu_river", seed=0, num_hands=4, max_raises=3)
    sg = wl.AbiSubgame(cfg)
    td = ssg.tree_struct(200)()
    b = (ctypes.c_int * 5)(*cfg["board"])
    s = (ctypes.c_float * 2)(*cfg["bet_sizes"])
    o = (ctypes.c_int * 2)(0, 1)
    assert sg.lib.ss_build_tree(b, 5, 100, 400, s, 2, 2, o, 1, 0, ctypes.byref(td)) == 0
    assert td.num_nodes == sg.td.num_nodes == 75
    sg.lib.ss_free_tree(ctypes.byref(td))
    assert td.num_nodes == 0 and not td.nodes
    sg.free()


def _solve_rc(sg, iters=1):
    rc, _ = sg.solve(iters)
    return rc, ssg.last_error(sg.lib)


def test_rejects_bad_cards():
    cfg = wl.config("hu_river", seed=1, num_hands=6)
    sg = wl.AbiSubgame(cfg)
    sg.td.hands[0][2][0] = 60
    rc, msg = _solve_rc(sg)
    assert rc == -1 and "distinct cards" in msg
    sg.td.hands[0][2][0] = sg.td.hands[0][2][1]
    rc, msg = _solve_rc(sg)
    assert rc == -1
    sg.free()


def test_rejects_too_many_hands_for_the_build():
    cfg = wl.config("hu_river", seed=1, num_hands=6)
    sg = wl.AbiSubgame(cfg, max_hands=200)
    sg.td.num_hands[1] = 201
    rc, msg = _solve_rc(sg)
    assert rc == -1 and "SS_MAX_HANDS" in msg
    sg.free()


def test_rejects_malformed_tree():
    cfg = wl.config("hu_river", seed=1, num_hands=6)
    sg = wl.AbiSubgame(cfg)
    first = sg.td.nodes[0].first_child
    sg.td.children[first + 1] = sg.td.children[first]  # a node reached twice
    rc, msg = _solve_rc(sg)
    assert rc == -1 and "tree" in msg
    sg.free()
    sg = wl.AbiSubgame(cfg)
    sg.td.nodes[0].num_children = 9
    rc, msg = _solve_rc(sg)
    assert rc == -1 and "actions" in msg
    sg.free()


def test_rejects_leaf_index_beyond_leaf_values():
    cfg = wl.config("turn3", seed=1, num_hands=5, bet_sizes=[1.0], max_raises=1)
    sg = wl.AbiSubgame(cfg)
    sg.set_leaf_values(wl.leaf_values_for(cfg, sg.num_leaves))
    sg.td.num_leaves = 3
    rc, msg = _solve_rc(sg)
    assert rc == -1 and "leaf_idx" in msg
    sg.free()


def test_rejects_empty_ranges_and_bad_iterations():
    cfg = wl.config("hu_river", seed=1, num_hands=6)
    sg = wl.AbiSubgame(cfg)
    rc, msg = _solve_rc(sg, iters=-3)
    assert rc == -1
    sg.td.num_hands[0] = 0
    sg.td.num_hands[1] = 0
    rc, msg = _solve_rc(sg)
    assert rc == -1 and "empty" in msg
    sg.free()


def test_large_multiway_enumeration_is_refused():
    """Terminals that still need enumeration at full range size -- the
    6-player river's folds with five counted opponents and its 4+-way
    showdowns -- are refused with SS_ERR_UNSUPPORTED instead of running for
    hours."""
    cfg = wl.config("river6", seed=0)
    sg = wl.AbiSubgame(cfg, max_hands=1326)
    rc, msg = _solve_rc(sg)
    assert rc == -4 and "tuple visits" in msg
    sg.free()


@pytest.mark.skipif(HAVE_GPU, reason="checks the behaviour without a GPU")
def test_no_cpu_fallback_without_gpu():
    cfg = wl.config("hu_river", seed=1, num_hands=6)
    sg = wl.AbiSubgame(cfg)
    rc, msg = _solve_rc(sg)
    assert rc == -5 and "no CUDA device" in msg
    sg.free()


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    monkeypatch.setattr(ssg, "LIB_DIR", str(tmp_path))
    monkeypatch.setattr(ssg, "_LIBS", {})
    with pytest.raises(FileNotFoundError):
        ssg.load_library(200)


def test_python_wrapper_tree_and_labels():
    s = ssg.StreetSolverGPU(board=["Qs", "As", "2d", "7h", "4c"], oop_range="AhKh,QhQc,JhTh,6h5h,3c3d",
                            ip_range="AcKc,8c8d,Tc9c,KhJh,2h2c", pot_bb=10.0, stack_bb=50.0,
                            bet_sizes=[0.33, 0.75])
    labels = ssg._build_labels_at_node(s._tree, 0)
    assert labels[0] == "Check" and labels[1].startswith("Bet ")
    s.set_frozen_actions(["Check"], hero_player=0)
    fz = np.ctypeslib.as_array(s._frozen_arr)
    assert fz[0] == 0 and (fz[1:] == -1).all()
    s.free()
    s.free()  # idempotent, no double free


def test_range_parser():
    from cards import card_to_int, int_to_card, parse_range_string
    assert card_to_int("Ah") == 50 and int_to_card(50) == "Ah" and card_to_int("2c") == 0
    assert len(parse_range_string("AA")) == 6
    assert len(parse_range_string("AKs")) == 4
    assert len(parse_range_string("AKo")) == 12
    assert len(parse_range_string("AA,AA,AhKh:0.5")) == 7
    combos = parse_range_string("AhKh:0.5")
    assert combos == [(card_to_int("Kh"), card_to_int("Ah"), 0.5)]
    with pytest.raises(ValueError):
        card_to_int("Xx")


def test_wrapper_trims_ranges_to_the_build_width():
    full = ",".join(["22", "33", "44", "55", "66", "77", "88", "99", "TT", "JJ", "QQ", "KK", "AA",
                     "AKs", "AQs", "AJs", "ATs", "KQs", "KJs", "QJs", "AKo", "AQo", "AJo", "KQo",
                     "KJo", "QJo", "JTs", "T9s", "98s", "87s", "76s", "65s", "ATo", "KTo", "QTo",
                     "JTo", "T9o", "98o", "87o", "76o"])
    s = ssg.StreetSolverGPU(board=["2s", "7d", "Jc", "Kh", "3s"], oop_range=full, ip_range=full,
                            pot_bb=5, stack_bb=20, bet_sizes=[1.0])
    assert all(len(h) <= 200 for h in s.player_hands)
    s.free()
    w = ssg.StreetSolverGPU(board=["2s", "7d", "Jc", "Kh", "3s"], oop_range=full, ip_range=full,
                            pot_bb=5, stack_bb=20, bet_sizes=[1.0], max_hands=1326)
    assert len(w.player_hands[0]) > 200
    w.free()


def test_wrapper_strategy_readout_on_a_given_output():
    # the reader of the reference module (street_solver_gpu.py:375-548) over
    # a synthetic output block: root strategy, the walk along action labels,
    # the per-hand average strategy map and the 0.001 cut
    s = ssg.StreetSolverGPU(board=["Qs", "As", "2d", "7h", "4c"], oop_range="AhKh,QhQc,JhTh",
                            ip_range="AcKc,8c8d", pot_bb=10.0, stack_bb=50.0, bet_sizes=[0.75])
    t = s._tree
    nd = t.num_decision_nodes
    ids = np.array([t.decision_node_indices[i] for i in range(nd)], np.int32)
    mh = s._max_hands
    avg = np.zeros((nd, 8, mh), np.float32)
    for di, nidx in enumerate(ids):
        na = t.nodes[int(nidx)].num_children
        for a in range(na):
            avg[di, a, :] = (a + 1) / (na * (na + 1) / 2)
    avg[0, 0, 1] = 0.0005                       # below the reader's cut
    nh0 = len(s.player_hands[0])
    na0 = t.nodes[0].num_children
    rs = np.full((na0, nh0), 1.0 / na0, np.float32)
    rev = np.zeros(mh, np.float32)
    keep = (avg, ids, rs, rev)
    o = ssg.SSOutput()
    o.root_strategy = rs.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    o.root_num_actions = na0
    o.root_player = 0
    o.root_ev = rev.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    o.avg_strategies = avg.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    o.avg_strategy_node_ids = ids.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
    o.num_avg_nodes = nd
    o.num_players_out = 2
    o.max_hands = mh
    s._output, s._solved = o, True
    try:
        labels0 = ssg._build_labels_at_node(t, 0)
        root = s.get_strategy(0, hand_idx=0)
        assert set(root) == set(labels0) and abs(sum(root.values()) - 1.0) < 1e-6
        # player 1 after "Check": the row of the child node
        child = t.children[t.nodes[0].first_child + labels0.index("Check")]
        di = int(np.nonzero(ids == child)[0][0])
        got = s.get_strategy(1, hand_idx=1, frozen_actions=["check"])
        labels1 = ssg._build_labels_at_node(t, child)
        assert got == {labels1[a]: float(avg[di, a, 1]) for a in range(len(labels1))}
        # player 0's first decision row, hand 1: the action under the cut is left out
        amap = s.get_avg_strategy(0)
        c0, c1, _ = s.player_hands[0][1]
        row = amap[(min(c0, c1), max(c0, c1))]
        assert labels0[0] not in row and set(row) == set(labels0[1:])
        assert s.get_avg_strategy_probs(0, labels0[0])[(min(c0, c1), max(c0, c1))] == 0.0
    finally:
        s._output, s._solved = ssg.SSOutput(), False   # synthetic buffers are not the library's
        del keep
        s.free()
