"""Python side of the multi-street (flop through river) two-player solver.

ctypes mirrors of include/flop_solve.h (the reference's flop_solve.cuh:45-114
layouts, as its callers bench/test_gpu_full_flop.py and precompute/run_all.py
declare them) and a small driver: build the tree, fill the ranges, solve,
read the outputs as numpy arrays, free.  The entry points live in this
repository's libstreet_solve(_wide).so; there is no CPU fallback (a missing
library raises FileNotFoundError, a failed call RuntimeError with the
library's message).
"""
import ctypes

import numpy as np

try:
    import street_solver_gpu as ssg
except ImportError:  # imported as part of a package
    from . import street_solver_gpu as ssg

FS_MAX_HANDS = 200
FS_MAX_ACTIONS = 6
NODE_DECISION, NODE_FOLD, NODE_SHOWDOWN, NODE_CHANCE = 0, 1, 2, 3


class FSNode(ctypes.Structure):
    _fields_ = [("type", ctypes.c_int), ("player", ctypes.c_int), ("num_children", ctypes.c_int),
                ("first_child", ctypes.c_int), ("pot", ctypes.c_int), ("bets", ctypes.c_int * 2),
                ("board_cards", ctypes.c_int * 5), ("num_board", ctypes.c_int)]


class FSTreeData(ctypes.Structure):
    _fields_ = [("nodes", ctypes.POINTER(FSNode)), ("children", ctypes.POINTER(ctypes.c_int)),
                ("num_nodes", ctypes.c_int), ("num_children_total", ctypes.c_int),
                ("hands", ((ctypes.c_int * 2) * FS_MAX_HANDS) * 2),
                ("weights", (ctypes.c_float * FS_MAX_HANDS) * 2),
                ("num_hands", ctypes.c_int * 2),
                ("level_order", ctypes.POINTER(ctypes.c_int)), ("node_depth", ctypes.POINTER(ctypes.c_int)),
                ("max_depth", ctypes.c_int),
                ("decision_node_indices", ctypes.POINTER(ctypes.c_int)), ("num_decision_nodes", ctypes.c_int),
                ("showdown_node_indices", ctypes.POINTER(ctypes.c_int)), ("num_showdown_nodes", ctypes.c_int)]


class FSOutput(ctypes.Structure):
    _fields_ = [("root_strategy", ctypes.POINTER(ctypes.c_float)), ("root_num_actions", ctypes.c_int),
                ("root_player", ctypes.c_int), ("root_ev", ctypes.POINTER(ctypes.c_float)),
                ("all_avg_strategies", ctypes.POINTER(ctypes.c_float)),
                ("all_cfv", ctypes.POINTER(ctypes.c_float)), ("max_hands", ctypes.c_int),
                ("turn_root_indices", ctypes.POINTER(ctypes.c_int)),
                ("turn_root_cards", ctypes.POINTER(ctypes.c_int)), ("num_turn_roots", ctypes.c_int)]


def bind(lib):
    """ctypes signatures of the fs_* entry points of a library (this
    repository's, or the reference's own build, which has the same ABI)."""
    T, O = ctypes.POINTER(FSTreeData), ctypes.POINTER(FSOutput)
    lib.fs_build_tree.restype = ctypes.c_int
    lib.fs_build_tree.argtypes = [ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.c_int,
                                  ctypes.POINTER(ctypes.c_float), ctypes.c_int, T]
    lib.fs_solve_gpu.restype = ctypes.c_int
    lib.fs_solve_gpu.argtypes = [T, ctypes.c_int, O]
    if hasattr(lib, "fs_solve_gpu_extract_all"):
        lib.fs_solve_gpu_extract_all.restype = ctypes.c_int
        lib.fs_solve_gpu_extract_all.argtypes = [T, ctypes.c_int, O]
    lib.fs_free_tree.restype = None
    lib.fs_free_tree.argtypes = [T]
    lib.fs_free_output.restype = None
    lib.fs_free_output.argtypes = [O]
    return lib


def tree_arrays(td):
    """(nodes [N, 13] int32, children, level_order, node_depth, decision ids, showdown ids)."""
    n = td.num_nodes
    nodes = np.ctypeslib.as_array(ctypes.cast(td.nodes, ctypes.POINTER(ctypes.c_int)), shape=(n * 13,))
    ch = np.ctypeslib.as_array(td.children, shape=(max(td.num_children_total, 1),))[:td.num_children_total]
    lo = np.ctypeslib.as_array(td.level_order, shape=(n,))
    nd = np.ctypeslib.as_array(td.node_depth, shape=(n,))
    dec = np.ctypeslib.as_array(td.decision_node_indices, shape=(max(td.num_decision_nodes, 1),))[
        :td.num_decision_nodes]
    sd = np.ctypeslib.as_array(td.showdown_node_indices, shape=(max(td.num_showdown_nodes, 1),))[
        :td.num_showdown_nodes]
    return (nodes.reshape(n, 13).copy(), ch.copy(), lo.copy(), nd.copy(), dec.copy(), sd.copy())


class FlopSubgame:
    """One flop-through-river subgame driven through a library's fs_* ABI."""

    def __init__(self, lib, flop, pot, stack, bet_sizes, hands, weights):
        self.lib = bind(lib)
        self.td = FSTreeData()
        b = (ctypes.c_int * 3)(*flop)
        s = (ctypes.c_float * max(len(bet_sizes), 1))(*bet_sizes)
        rc = self.lib.fs_build_tree(b, int(pot), int(stack), s, len(bet_sizes), ctypes.byref(self.td))
        if rc != 0:
            raise RuntimeError(f"fs_build_tree failed ({rc}): {ssg.last_error(lib) if hasattr(lib, 'ss_last_error') else ''}")
        for p in range(2):
            n = len(hands[p])
            if n > FS_MAX_HANDS:
                raise ValueError("at most 200 hands per player")
            self.td.num_hands[p] = n
            for i in range(n):
                self.td.hands[p][i][0], self.td.hands[p][i][1] = int(hands[p][i][0]), int(hands[p][i][1])
                self.td.weights[p][i] = float(weights[p][i])
        self.nh = [len(hands[0]), len(hands[1])]

    def solve(self, iterations, extract=False):
        out = FSOutput()
        fn = self.lib.fs_solve_gpu_extract_all if extract else self.lib.fs_solve_gpu
        rc = fn(ctypes.byref(self.td), int(iterations), ctypes.byref(out))
        if rc != 0:
            msg = ssg.last_error(self.lib) if hasattr(self.lib, "ss_last_error") else ""
            raise RuntimeError(f"fs solve failed ({rc}): {msg}")
        na, rp = out.root_num_actions, out.root_player
        res = {"root_player": rp, "root_num_actions": na,
               "root_strategy": np.ctypeslib.as_array(out.root_strategy, shape=(na * self.nh[rp],)).copy().reshape(
                   na, self.nh[rp])}
        if extract:
            n, mh = self.td.num_nodes, out.max_hands
            res["max_hands"] = mh
            res["all_avg_strategies"] = np.ctypeslib.as_array(
                out.all_avg_strategies, shape=(n * FS_MAX_ACTIONS * mh,)).copy().reshape(n, FS_MAX_ACTIONS, mh)
            res["all_cfv"] = np.ctypeslib.as_array(out.all_cfv, shape=(n * mh,)).copy().reshape(n, mh)
            k = out.num_turn_roots
            res["turn_root_indices"] = np.ctypeslib.as_array(out.turn_root_indices, shape=(max(k, 1),))[:k].copy()
            res["turn_root_cards"] = np.ctypeslib.as_array(out.turn_root_cards, shape=(max(k, 1),))[:k].copy()
        self.lib.fs_free_output(ctypes.byref(out))
        return res

    def free(self):
        if self.td.nodes:
            self.lib.fs_free_tree(ctypes.byref(self.td))
