"""ss_solve_gpu_noalloc: the solve for callers that cannot allocate GPU memory
(their device memory belongs to another allocator, or their serving path
forbids allocation).  It keeps all device state in the library's static
device array and writes into output arrays the caller provides.  Through the
C ABI it must match ss_solve_gpu within the parity tolerance on two calls in
a row (the second call reuses the array the first one left behind), and it
must refuse a subgame too large for the array.  This file sorts last so that
a run stopping at the first failure has run every other test before it."""
import ctypes

import numpy as np
import pytest

import street_solver_gpu as ssg
import workloads as wl

STRAT_ATOL = 1e-4
EV_RTOL = 1e-4


def caller_buffers(sg):
    """Output arrays owned by the caller, sized from the built tree."""
    td = sg.td
    np_ = td.num_players_field
    mh = int(max(td.num_hands[p] for p in range(np_)))
    root = td.nodes[0]
    na, nh_root = root.num_children, td.num_hands[root.player]
    bufs = {
        "rs": np.full(na * nh_root, -7.0, np.float32),
        "rev": np.full(np_ * mh, -7.0, np.float32),
        "avg": np.full(td.num_decision_nodes * 8 * mh, -7.0, np.float32),
        "ids": np.full(td.num_decision_nodes, -7, np.int32),
    }
    out = ssg.SSOutput()
    fp = ctypes.POINTER(ctypes.c_float)
    out.root_strategy = bufs["rs"].ctypes.data_as(fp)
    out.root_ev = bufs["rev"].ctypes.data_as(fp)
    out.avg_strategies = bufs["avg"].ctypes.data_as(fp)
    out.avg_strategy_node_ids = bufs["ids"].ctypes.data_as(ctypes.POINTER(ctypes.c_int))
    return out, bufs, (na, nh_root, mh)


def noalloc_solve(sg, iters):
    out, bufs, (na, nh_root, mh) = caller_buffers(sg)
    sg.lib.ss_solve_gpu_noalloc.restype = ctypes.c_int
    rc = sg.lib.ss_solve_gpu_noalloc(ctypes.byref(sg.td), iters, ctypes.byref(out))
    assert rc == 0, ssg.last_error(sg.lib)
    nd = sg.td.num_decision_nodes
    return {
        "root_strategy": bufs["rs"].reshape(na, nh_root),
        "root_ev": bufs["rev"][:mh],
        "avg_strategies": bufs["avg"].reshape(nd, 8, mh),
        "avg_node_ids": bufs["ids"],
        "root_player": out.root_player,
        "root_num_actions": out.root_num_actions,
    }


def same(a, b):
    assert np.array_equal(a["avg_node_ids"], b["avg_node_ids"])
    assert a["root_player"] == b["root_player"] and a["root_num_actions"] == b["root_num_actions"]
    assert np.abs(a["avg_strategies"] - b["avg_strategies"]).max() <= STRAT_ATOL
    assert np.abs(a["root_strategy"] - b["root_strategy"]).max() <= STRAT_ATOL
    scale = max(float(np.abs(b["root_ev"]).max()), 1e-30)
    assert np.abs(a["root_ev"] - b["root_ev"]).max() / scale <= EV_RTOL


@pytest.mark.gpu
@pytest.mark.parametrize("name,nh,iters", [("hu_river", 120, 40), ("turn3", 10, 6)])
def test_noalloc_matches_solve_twice(name, nh, iters):
    over = {"bet_sizes": [0.75], "max_raises": 2} if name == "turn3" else {}
    cfg = wl.config(name, seed=31, num_hands=nh, **over)
    sg = wl.AbiSubgame(cfg)
    sg.set_leaf_values(wl.leaf_values_for(cfg, sg.num_leaves))
    rc, ref = sg.solve(iters)
    assert rc == 0, ssg.last_error(sg.lib)
    first = noalloc_solve(sg, iters)
    second = noalloc_solve(sg, iters)
    same(first, ref)
    same(second, ref)
    sg.free()


@pytest.mark.gpu
def test_noalloc_interleaved_subgames():
    """A heads-up river, then a 3-player turn with other leaf values, then
    the river again, all in the one shared array: each call must rewrite what
    it reads, so every result equals its own ss_solve_gpu solve."""
    river = wl.config("hu_river", seed=41, num_hands=90)
    turn = wl.config("turn3", seed=42, num_hands=12, bet_sizes=[0.75], max_raises=2)
    subs = []
    for cfg, seed in ((river, 0), (turn, 777)):
        sg = wl.AbiSubgame(cfg)
        sg.set_leaf_values(wl.leaf_values_for(cfg, sg.num_leaves, seed_offset=seed + 1000))
        subs.append(sg)
    refs = []
    for sg in subs:
        rc, ref = sg.solve(8)
        assert rc == 0, ssg.last_error(sg.lib)
        refs.append(ref)
    for k in (0, 1, 0):
        same(noalloc_solve(subs[k], 8), refs[k])
    for sg in subs:
        sg.free()


@pytest.mark.gpu
def test_noalloc_refuses_oversized_subgame():
    cfg = wl.config("turn3", seed=0)  # ~600 MB of device state
    sg = wl.AbiSubgame(cfg, max_hands=1326)
    sg.set_leaf_values(wl.leaf_values_for(cfg, sg.num_leaves))
    out, _, _ = caller_buffers(sg)
    sg.lib.ss_solve_gpu_noalloc.restype = ctypes.c_int
    rc = sg.lib.ss_solve_gpu_noalloc(ctypes.byref(sg.td), 1, ctypes.byref(out))
    assert rc == -3 and "static arena" in ssg.last_error(sg.lib)
    sg.free()
