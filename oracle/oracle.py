"""ctypes front end of the oracle and of the reference builds in oracle/_ref/.

TEST INFRASTRUCTURE ONLY.  Only tests/, the smoke check in __graft_entry__.py
and the CPU-baseline leg of bench.py import this module, and only as the
checker (or, for bench.py, as the timed CPU baseline).  The product library
never imports, links or calls anything under oracle/.

Two back ends with one Python interface:
  * Oracle      -- liboracle.so, the C restatement in this directory
                   (ss_oracle.c / ss_oracle_impl.h / oracle_eval.h).
  * RefShim     -- oracle/_ref/ref_h{H}_r{R}/libref_street_solve_cpu.so, the
                   reference src/cuda/street_solve.cu compiled for the CPU by
                   oracle/build_ref.py (its own kernels, run as host loops).
Both return solve outputs in the reference layout (street_solve.cu:1563-1612):
root_strategy [na][nh_root], root_ev [max_h], avg_strategies
[num_dec][8][max_h] and avg_node_ids [num_dec].
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
MAX_PLAYERS = 6
MAX_ACTIONS = 8
NODE_DECISION, NODE_FOLD, NODE_SHOWDOWN, NODE_LEAF = 0, 1, 2, 4

NODE_FIELDS = [
    ("type", ctypes.c_int), ("player", ctypes.c_int), ("num_children", ctypes.c_int),
    ("first_child", ctypes.c_int), ("pot", ctypes.c_int),
    ("bets", ctypes.c_int * MAX_PLAYERS), ("board_cards", ctypes.c_int * 5),
    ("num_board", ctypes.c_int), ("leaf_idx", ctypes.c_int), ("fold_player", ctypes.c_int),
    ("num_players", ctypes.c_int), ("active_players", ctypes.c_int * MAX_PLAYERS),
]


class Node(ctypes.Structure):
    _fields_ = NODE_FIELDS


NODE_INTS = ctypes.sizeof(Node) // 4  # 26


class OrcTree(ctypes.Structure):
    _fields_ = [
        ("nodes", ctypes.POINTER(Node)), ("children", ctypes.POINTER(ctypes.c_int)),
        ("num_nodes", ctypes.c_int), ("num_children_total", ctypes.c_int),
        ("num_leaves", ctypes.c_int), ("num_players", ctypes.c_int),
        ("is_river", ctypes.c_int), ("starting_pot", ctypes.c_int),
        ("effective_stack", ctypes.c_int), ("board", ctypes.c_int * 5),
        ("num_board", ctypes.c_int), ("level_order", ctypes.POINTER(ctypes.c_int)),
        ("node_depth", ctypes.POINTER(ctypes.c_int)), ("max_depth", ctypes.c_int),
    ]


def _f32p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float)) if a is not None else None


def _f64p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if a is not None else None


def _i32p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int)) if a is not None else None


class Tree:
    """A built betting tree as numpy arrays (node fields as an [N, 23] int
    matrix in SSNode order, children, BFS order, depths)."""

    def __init__(self, nodes, children, level_order, node_depth, max_depth, num_leaves,
                 num_players, is_river, starting_pot, effective_stack, board):
        self.nodes = nodes
        self.children = children
        self.level_order = level_order
        self.node_depth = node_depth
        self.max_depth = max_depth
        self.num_leaves = num_leaves
        self.num_players = num_players
        self.is_river = is_river
        self.starting_pot = starting_pot
        self.effective_stack = effective_stack
        self.board = list(board)

    @property
    def num_nodes(self):
        return self.nodes.shape[0]

    def col(self, name):
        off = 0
        for fname, ftype in NODE_FIELDS:
            width = ctypes.sizeof(ftype) // 4
            if fname == name:
                return self.nodes[:, off] if width == 1 else self.nodes[:, off:off + width]
            off += width
        raise KeyError(name)

    def decision_nodes(self):
        return np.nonzero(self.col("type") == NODE_DECISION)[0].astype(np.int32)


def _tree_from_orc(t):
    n = t.num_nodes
    raw = np.ctypeslib.as_array(ctypes.cast(t.nodes, ctypes.POINTER(ctypes.c_int)),
                                shape=(n * NODE_INTS,)).reshape(n, NODE_INTS).copy()
    ch = np.ctypeslib.as_array(t.children, shape=(max(t.num_children_total, 1),))[
        :t.num_children_total].copy()
    lo = np.ctypeslib.as_array(t.level_order, shape=(n,)).copy()
    nd = np.ctypeslib.as_array(t.node_depth, shape=(n,)).copy()
    return Tree(raw, ch, lo, nd, t.max_depth, t.num_leaves, t.num_players, t.is_river,
                t.starting_pot, t.effective_stack, list(t.board)[:t.num_board])


def _tree_to_orc(tree):
    """Owned ctypes OrcTree view of a Tree (keeps the numpy buffers alive)."""
    t = OrcTree()
    keep = []
    nodes = np.ascontiguousarray(tree.nodes, dtype=np.int32)
    ch = np.ascontiguousarray(tree.children, dtype=np.int32)
    lo = np.ascontiguousarray(tree.level_order, dtype=np.int32)
    nd = np.ascontiguousarray(tree.node_depth, dtype=np.int32)
    keep += [nodes, ch, lo, nd]
    t.nodes = ctypes.cast(nodes.ctypes.data, ctypes.POINTER(Node))
    t.children = _i32p(ch)
    t.num_nodes = nodes.shape[0]
    t.num_children_total = ch.shape[0]
    t.num_leaves = tree.num_leaves
    t.num_players = tree.num_players
    t.is_river = tree.is_river
    t.starting_pot = tree.starting_pot
    t.effective_stack = tree.effective_stack
    for i, c in enumerate(tree.board[:5]):
        t.board[i] = c
    t.num_board = len(tree.board)
    t.level_order = _i32p(lo)
    t.node_depth = _i32p(nd)
    t.max_depth = tree.max_depth
    return t, keep


class Oracle:
    """The C restatement (liboracle.so)."""

    def __init__(self, path=None):
        self.lib = ctypes.CDLL(path or _default_oracle_path())
        L = self.lib
        L.orc_build_tree.restype = ctypes.c_int
        L.orc_eval7_cards.restype = ctypes.c_uint32
        L.orc_solve_f32.restype = ctypes.c_int
        L.orc_solve_f64.restype = ctypes.c_int
        L.orc_solve_f64_closed.restype = ctypes.c_int
        L.orc_exploitability.restype = ctypes.c_double
        L.orc_profile_cfv.restype = ctypes.c_int

    def build_tree(self, board, starting_pot, effective_stack, bet_sizes, num_players,
                   acting_order=None, is_river=None, use_cont_strats=True, max_raises=3):
        if acting_order is None:
            acting_order = list(range(num_players))
        if is_river is None:
            is_river = len(board) == 5
        t = OrcTree()
        b = (ctypes.c_int * max(len(board), 1))(*board)
        s = (ctypes.c_float * max(len(bet_sizes), 1))(*bet_sizes)
        o = (ctypes.c_int * len(acting_order))(*acting_order)
        rc = self.lib.orc_build_tree(b, len(board), starting_pot, effective_stack, s,
                                     len(bet_sizes), num_players, o, int(bool(is_river)),
                                     int(bool(use_cont_strats and not is_river)), max_raises,
                                     ctypes.byref(t))
        if rc != 0:
            raise RuntimeError("orc_build_tree failed")
        tree = _tree_from_orc(t)
        self.lib.orc_free_tree(ctypes.byref(t))
        return tree

    def eval7(self, cards7):
        a = (ctypes.c_int * 7)(*cards7)
        return int(self.lib.orc_eval7_cards(a))

    def solve(self, tree, hands, weights, num_hands, iterations, leaf_values=None,
              frozen=None, precision="f32", want_state=False):
        hands = np.ascontiguousarray(hands, dtype=np.int32)
        weights = np.ascontiguousarray(weights, dtype=np.float32)
        nh = np.ascontiguousarray(num_hands, dtype=np.int32)
        np_, max_h = weights.shape
        assert hands.shape == (np_, max_h, 2) and max_h == int(nh.max())
        lv = None if leaf_values is None else np.ascontiguousarray(leaf_values, dtype=np.float32)
        fz = None if frozen is None else np.ascontiguousarray(frozen, dtype=np.int32)
        dt = np.float32 if precision == "f32" else np.float64
        ptr = _f32p if precision == "f32" else _f64p
        nodes_t = tree.col("type")
        root = tree.nodes[0]
        root_player = int(tree.col("player")[0])
        na = int(tree.col("num_children")[0])
        nh_root = int(nh[root_player]) if root_player >= 0 else 0
        ndec = int((nodes_t == NODE_DECISION).sum())
        rs = np.zeros(max(na * nh_root, 1), dt)
        rev = np.zeros(max_h, dt)
        avg = np.zeros(ndec * MAX_ACTIONS * max_h, dt)
        ids = np.zeros(max(ndec, 1), np.int32)
        N = tree.num_nodes
        reg = np.zeros(N * MAX_ACTIONS * max_h, dt) if want_state else None
        ssum = np.zeros(N * MAX_ACTIONS * max_h, dt) if want_state else None
        t, keep = _tree_to_orc(tree)
        fn = {"f32": self.lib.orc_solve_f32, "f64": self.lib.orc_solve_f64,
              "f64_closed": self.lib.orc_solve_f64_closed}[precision]
        rc = fn(ctypes.byref(t), _i32p(hands), _f32p(weights), _i32p(nh), _f32p(lv), _i32p(fz),
                iterations, ptr(rs), ptr(rev), ptr(avg), _i32p(ids), ptr(reg), ptr(ssum))
        del keep, root
        if rc != 0:
            raise RuntimeError("orc_solve failed")
        out = {
            "root_strategy": rs[:na * nh_root].reshape(na, nh_root),
            "root_ev": rev,
            "avg_strategies": avg.reshape(ndec, MAX_ACTIONS, max_h),
            "avg_node_ids": ids[:ndec],
            "root_player": root_player,
            "root_num_actions": na,
        }
        if want_state:
            out["regrets"] = reg.reshape(N, MAX_ACTIONS, max_h)
            out["strategy_sum"] = ssum.reshape(N, MAX_ACTIONS, max_h)
        return out

    def exploitability(self, tree, hands, weights, num_hands, avg_strategies,
                       leaf_values=None, frozen=None):
        hands = np.ascontiguousarray(hands, dtype=np.int32)
        weights = np.ascontiguousarray(weights, dtype=np.float32)
        nh = np.ascontiguousarray(num_hands, dtype=np.int32)
        avg = np.ascontiguousarray(avg_strategies, dtype=np.float32)
        lv = None if leaf_values is None else np.ascontiguousarray(leaf_values, dtype=np.float32)
        fz = None if frozen is None else np.ascontiguousarray(frozen, dtype=np.int32)
        np_ = weights.shape[0]
        br = np.zeros(np_, np.float64)
        cur = np.zeros(np_, np.float64)
        z = ctypes.c_double(0)
        t, keep = _tree_to_orc(tree)
        nc = self.lib.orc_exploitability(ctypes.byref(t), _i32p(hands), _f32p(weights), _i32p(nh),
                                         _f32p(lv), _i32p(fz), _f32p(avg), _f64p(br), _f64p(cur),
                                         ctypes.byref(z))
        del keep
        return {"nashconv": float(nc), "br_value": br, "cur_value": cur,
                "deal_mass": float(z.value),
                "exploitability_pct": float(nc) / np_ / tree.starting_pot * 100.0}

    def profile_cfv(self, tree, hands, weights, num_hands, avg_strategies, traverser, mode,
                    leaf_values=None, frozen=None):
        hands = np.ascontiguousarray(hands, dtype=np.int32)
        weights = np.ascontiguousarray(weights, dtype=np.float32)
        nh = np.ascontiguousarray(num_hands, dtype=np.int32)
        avg = np.ascontiguousarray(avg_strategies, dtype=np.float32)
        lv = None if leaf_values is None else np.ascontiguousarray(leaf_values, dtype=np.float32)
        fz = None if frozen is None else np.ascontiguousarray(frozen, dtype=np.int32)
        out = np.zeros(weights.shape[1], np.float64)
        t, keep = _tree_to_orc(tree)
        rc = self.lib.orc_profile_cfv(ctypes.byref(t), _i32p(hands), _f32p(weights), _i32p(nh),
                                      _f32p(lv), _i32p(fz), _f32p(avg), traverser, mode,
                                      _f64p(out))
        del keep
        if rc != 0:
            raise RuntimeError("orc_profile_cfv failed")
        return out


def _default_oracle_path():
    path = os.path.join(HERE, "lib", "liboracle.so")
    if not os.path.exists(path):
        import importlib.util
        spec = importlib.util.spec_from_file_location("_oracle_build", os.path.join(HERE, "build.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        mod.build()
    return path


# --------------------------------------------------------------------------
# Reference builds (oracle/_ref)
# --------------------------------------------------------------------------

def ref_tree_struct(max_hands):
    """ctypes mirror of the reference SSTreeData for a given SS_MAX_HANDS
    (src/cuda/street_solve.cuh:69-122)."""

    class RefTree(ctypes.Structure):
        _fields_ = [
            ("nodes", ctypes.POINTER(Node)), ("children", ctypes.POINTER(ctypes.c_int)),
            ("num_nodes", ctypes.c_int), ("num_children_total", ctypes.c_int),
            ("num_players", ctypes.c_int),
            ("hands", ((ctypes.c_int * 2) * max_hands) * MAX_PLAYERS),
            ("weights", (ctypes.c_float * max_hands) * MAX_PLAYERS),
            ("num_hands", ctypes.c_int * MAX_PLAYERS), ("board", ctypes.c_int * 5),
            ("num_board", ctypes.c_int), ("leaf_values", ctypes.POINTER(ctypes.c_float)),
            ("num_leaves", ctypes.c_int), ("level_order", ctypes.POINTER(ctypes.c_int)),
            ("node_depth", ctypes.POINTER(ctypes.c_int)), ("max_depth", ctypes.c_int),
            ("decision_node_indices", ctypes.POINTER(ctypes.c_int)),
            ("num_decision_nodes", ctypes.c_int),
            ("showdown_node_indices", ctypes.POINTER(ctypes.c_int)),
            ("num_showdown_nodes", ctypes.c_int),
            ("leaf_node_indices", ctypes.POINTER(ctypes.c_int)), ("num_leaf_nodes", ctypes.c_int),
            ("fold_node_indices", ctypes.POINTER(ctypes.c_int)), ("num_fold_nodes", ctypes.c_int),
            ("starting_pot", ctypes.c_int), ("effective_stack", ctypes.c_int),
            ("is_river", ctypes.c_int), ("frozen_action", ctypes.POINTER(ctypes.c_int)),
        ]

    return RefTree


class RefOutput(ctypes.Structure):
    _fields_ = [
        ("root_strategy", ctypes.POINTER(ctypes.c_float)), ("root_num_actions", ctypes.c_int),
        ("root_player", ctypes.c_int), ("root_ev", ctypes.POINTER(ctypes.c_float)),
        ("avg_strategies", ctypes.POINTER(ctypes.c_float)),
        ("avg_strategy_node_ids", ctypes.POINTER(ctypes.c_int)), ("num_avg_nodes", ctypes.c_int),
        ("num_players", ctypes.c_int), ("max_hands", ctypes.c_int),
    ]


class RefStreetSolve:
    """The reference street_solve.cu through its own C ABI: the CPU-shim build
    (kind="cpu") or the stock sm_100a build (kind="gpu", 200 hands, 3 raises)."""

    def __init__(self, max_hands=200, max_raises=3, kind="cpu"):
        if kind == "cpu":
            path = os.path.join(REF_DIR, f"ref_h{max_hands}_r{max_raises}",
                                "libref_street_solve_cpu.so")
        else:
            assert (max_hands, max_raises) == (200, 3)
            path = os.path.join(REF_DIR, "libref_street_solve_gpu.so")
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.max_hands = max_hands
        self.lib = ctypes.CDLL(path)
        self.Tree = ref_tree_struct(max_hands)
        self.lib.ss_build_tree.restype = ctypes.c_int
        self.lib.ss_solve_gpu.restype = ctypes.c_int

    def build(self, board, starting_pot, effective_stack, bet_sizes, num_players,
              acting_order=None, is_river=None, use_cont_strats=True):
        if acting_order is None:
            acting_order = list(range(num_players))
        if is_river is None:
            is_river = len(board) == 5
        td = self.Tree()
        b = (ctypes.c_int * max(len(board), 1))(*board)
        s = (ctypes.c_float * max(len(bet_sizes), 1))(*bet_sizes)
        o = (ctypes.c_int * len(acting_order))(*acting_order)
        rc = self.lib.ss_build_tree(b, len(board), starting_pot, effective_stack, s,
                                    len(bet_sizes), num_players, o, int(bool(is_river)),
                                    int(bool(use_cont_strats and not is_river)), ctypes.byref(td))
        if rc != 0:
            raise RuntimeError("reference ss_build_tree failed")
        return td

    def tree(self, td):
        """Tree view (numpy) of a reference SSTreeData."""
        n = td.num_nodes
        raw = np.ctypeslib.as_array(ctypes.cast(td.nodes, ctypes.POINTER(ctypes.c_int)),
                                    shape=(n * NODE_INTS,)).reshape(n, NODE_INTS).copy()
        ch = np.ctypeslib.as_array(td.children, shape=(max(td.num_children_total, 1),))[
            :td.num_children_total].copy()
        lo = np.ctypeslib.as_array(td.level_order, shape=(n,)).copy()
        nd = np.ctypeslib.as_array(td.node_depth, shape=(n,)).copy()
        return Tree(raw, ch, lo, nd, td.max_depth, td.num_leaves, td.num_players, td.is_river,
                    td.starting_pot, td.effective_stack, list(td.board)[:td.num_board])

    def solve(self, td, hands, weights, num_hands, iterations, leaf_values=None, frozen=None):
        np_ = td.num_players
        for p in range(np_):
            td.num_hands[p] = int(num_hands[p])
            for h in range(int(num_hands[p])):
                td.hands[p][h][0] = int(hands[p][h][0])
                td.hands[p][h][1] = int(hands[p][h][1])
                td.weights[p][h] = float(weights[p][h])
        keep = []
        if leaf_values is not None:
            lv = np.ascontiguousarray(leaf_values, dtype=np.float32).ravel()
            keep.append(lv)
            td.leaf_values = _f32p(lv)
        if frozen is not None:
            fz = np.ascontiguousarray(frozen, dtype=np.int32)
            keep.append(fz)
            td.frozen_action = _i32p(fz)
        out = RefOutput()
        rc = self.lib.ss_solve_gpu(ctypes.byref(td), iterations, ctypes.byref(out))
        td.leaf_values = None
        td.frozen_action = None
        if rc != 0:
            raise RuntimeError("reference ss_solve_gpu failed")
        max_h = out.max_hands
        na, rp = out.root_num_actions, out.root_player
        nh_root = int(num_hands[rp])
        nd = out.num_avg_nodes
        res = {
            "root_strategy": np.ctypeslib.as_array(out.root_strategy, shape=(na * nh_root,))
            .copy().reshape(na, nh_root),
            "root_ev": np.ctypeslib.as_array(out.root_ev, shape=(np_ * max_h,)).copy()[:max_h],
            "avg_strategies": np.ctypeslib.as_array(out.avg_strategies,
                                                    shape=(nd * MAX_ACTIONS * max_h,))
            .copy().reshape(nd, MAX_ACTIONS, max_h),
            "avg_node_ids": np.ctypeslib.as_array(out.avg_strategy_node_ids, shape=(nd,)).copy(),
            "root_player": rp,
            "root_num_actions": na,
        }
        self.lib.ss_free_output(ctypes.byref(out))
        return res

    def free(self, td):
        td.leaf_values = None  # caller-owned; the reference would free() it
        self.lib.ss_free_tree(ctypes.byref(td))


class RefHandEval:
    """src/hand_eval.h through oracle/_ref/libref_handeval.so."""

    def __init__(self):
        self.lib = ctypes.CDLL(os.path.join(REF_DIR, "libref_handeval.so"))
        self.lib.ref_eval7.restype = ctypes.c_uint32

    def eval7_many(self, cards):
        cards = np.ascontiguousarray(cards, dtype=np.int32)
        out = np.zeros(cards.shape[0], np.uint32)
        self.lib.ref_eval7_many(_i32p(cards), ctypes.c_long(cards.shape[0]),
                                out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)))
        return out


def ref_available(max_hands=200, max_raises=3):
    return os.path.exists(os.path.join(REF_DIR, f"ref_h{max_hands}_r{max_raises}",
                                       "libref_street_solve_cpu.so"))


class RefSolverC:
    """src/solver.c, the reference's 2-player CPU Linear-CFR solver (built
    -O2 -fopenmp into oracle/_ref/libref_solver.so), through its own API
    (src/solver.h:140-187).  Its Solver struct holds fixed-size ranges
    (MAX_HANDS = 1326, about 32 KB); it is passed as an opaque zeroed block
    of SOLVER_BYTES.  Used as a CPU timing baseline only: its payoff, tie,
    averaging and discount rules differ from street_solve.cu's."""

    SOLVER_BYTES = 1 << 16

    def __init__(self):
        path = os.path.join(REF_DIR, "libref_solver.so")
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = ctypes.CDLL(path)
        ip, fp, vp = ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_float), ctypes.c_void_p
        self.lib.solver_init.restype = ctypes.c_int
        self.lib.solver_init.argtypes = [vp, ip, ctypes.c_int, ip, fp, ctypes.c_int, ip, fp, ctypes.c_int,
                                         ctypes.c_int, ctypes.c_int, fp, ctypes.c_int]
        self.lib.solver_solve.restype = ctypes.c_float
        self.lib.solver_solve.argtypes = [vp, ctypes.c_int, ctypes.c_float]
        self.lib.solver_free.restype = None
        self.lib.solver_free.argtypes = [vp]

    def solve(self, board, hands, weights, starting_pot, effective_stack, bet_sizes, iterations):
        """One solve (solver_init, solver_solve, solver_free); returns the
        seconds spent in solver_solve."""
        import time
        b = np.ascontiguousarray(board, dtype=np.int32)
        h = [np.ascontiguousarray(x, dtype=np.int32).reshape(-1, 2) for x in hands]
        w = [np.ascontiguousarray(x, dtype=np.float32) for x in weights]
        sz = np.ascontiguousarray(bet_sizes, dtype=np.float32)
        blk = ctypes.create_string_buffer(self.SOLVER_BYTES)
        rc = self.lib.solver_init(blk, _i32p(b), len(b), _i32p(h[0]), _f32p(w[0]), len(w[0]),
                                  _i32p(h[1]), _f32p(w[1]), len(w[1]), int(starting_pot), int(effective_stack),
                                  _f32p(sz), len(sz))
        if rc != 0:
            raise RuntimeError(f"solver_init failed ({rc})")
        try:
            t0 = time.perf_counter()
            self.lib.solver_solve(blk, int(iterations), ctypes.c_float(0.0))
            return time.perf_counter() - t0
        finally:
            self.lib.solver_free(blk)


def ref_solver_available():
    return os.path.exists(os.path.join(REF_DIR, "libref_solver.so"))


class FlopOracle:
    """The multi-street solve restated in C (fs_oracle.c, in liboracle.so):
    the reference's flop_solve.cu loop in float (its arithmetic and order,
    fused multiply-adds included) or double, on a tree from fs_build_tree."""

    def __init__(self, path=None):
        self.lib = ctypes.CDLL(path or _default_oracle_path())
        for f in ("fso_solve_f32", "fso_solve_f64"):
            getattr(self.lib, f).restype = ctypes.c_int

    def solve(self, nodes, children, node_depth, max_depth, hands, weights, nh, iterations, precision="f32",
              snapshots=(), full=True):
        """nodes [N, 13] int32 (FSNode fields), hands [2][200][2], weights
        [2][200]; returns root_strategy, all_avg_strategies [N][6][max_h] and
        all_cfv [N][max_h] (None without `full`), and root_snapshots {k: the
        root strategy after iteration k} for each k in `snapshots`."""
        nodes = np.ascontiguousarray(nodes, np.int32)
        children = np.ascontiguousarray(children, np.int32)
        nd = np.ascontiguousarray(node_depth, np.int32)
        hands = np.ascontiguousarray(hands, np.int32)
        weights = np.ascontiguousarray(weights, np.float32)
        nh = np.ascontiguousarray(nh, np.int32)
        N = nodes.shape[0]
        mh = int(nh.max())
        dt = np.float32 if precision == "f32" else np.float64
        ptr = _f32p if precision == "f32" else _f64p
        rp, na = int(nodes[0, 1]), int(nodes[0, 2])
        rs = np.zeros(max(na * int(nh[rp]), 1), dt)
        avg = np.zeros(N * 6 * mh, dt) if full else None
        cfv = np.zeros(N * mh, dt) if full else None
        snaps = np.ascontiguousarray([int(k) for k in snapshots] or [0], np.int32)
        sr = np.zeros(max(len(snapshots), 1) * max(na * int(nh[rp]), 1), dt)
        fn = self.lib.fso_solve_f32 if precision == "f32" else self.lib.fso_solve_f64
        rc = fn(_i32p(nodes), _i32p(children), N, _i32p(nd), int(max_depth), _i32p(hands), _f32p(weights),
                _i32p(nh), int(iterations), ptr(rs), ptr(avg) if full else None, ptr(cfv) if full else None,
                len(snapshots), _i32p(snaps), ptr(sr))
        if rc != 0:
            raise RuntimeError("fso_solve failed")
        k = na * int(nh[rp])
        return {"root_strategy": rs[:k].reshape(na, int(nh[rp])),
                "all_avg_strategies": avg.reshape(N, 6, mh) if full else None,
                "all_cfv": cfv.reshape(N, mh) if full else None,
                "root_snapshots": {int(s_): sr[j * k:(j + 1) * k].reshape(na, int(nh[rp]))
                                   for j, s_ in enumerate(snapshots)}}
