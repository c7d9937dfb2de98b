"""Seeded synthetic subgames with the shapes of the benchmark configurations,
and a direct C-ABI driver (build -> fill -> solve -> read -> free).

The configurations (sizes, bet sizes, raise caps, weight distributions) are
the ones the reference's benchmark plan quotes; inputs are synthetic and
seeded, there is no dataset:

  hu_river   2 players, 5-card board, all 1081 combos each, weights U(0,1),
             pot 100, stack 400, bets {0.5, 1.0} + all-in, 2 raises
  turn3      3 players, 4-card board, all 1128 combos each, weights U(0,1)
             with ~30% zeroed, pot 150, stack 500, bets {0.33, 0.75, 1.5}
             + all-in, 3 raises, continuation leaves with values N(0, 0.3 pot)
  river6     6 players, 5-card board, 1081 combos each, Dirichlet(0.3)-style
             sparse weights (40-70% zero), pot 300, stack 1000,
             bets {0.5, 1.0} + all-in, 2 raises
"""
import ctypes

import numpy as np

NODE_INTS = 26  # SSNode is 26 x int32

try:
    import street_solver_gpu as ssg
except ImportError:  # imported as part of a package
    from . import street_solver_gpu as ssg


def all_combos(board):
    deck = [c for c in range(52) if c not in set(board)]
    return [(a, b) for i, a in enumerate(deck) for b in deck[i + 1:]]


def make_ranges(rng, board, num_players, num_hands=None, weights="uniform", zero_frac=0.0):
    """Per player: hands [H, 2] int32 and weights [H] float32 over non-board
    combos (all of them when num_hands is None, else a random subset)."""
    combos = all_combos(board)
    hands, ws = [], []
    for _ in range(num_players):
        if num_hands is None or num_hands >= len(combos):
            sel = np.arange(len(combos))
        else:
            sel = np.sort(rng.choice(len(combos), num_hands, replace=False))
        h = np.array([combos[i] for i in sel], np.int32)
        if weights == "dirichlet":
            w = rng.gamma(0.3, 1.0, len(sel))
            w = w / w.max()
            zf = rng.uniform(0.4, 0.7)
            w[rng.random(len(sel)) < zf] = 0.0
        else:
            w = rng.uniform(0.0, 1.0, len(sel))
            if zero_frac > 0:
                w[rng.random(len(sel)) < zero_frac] = 0.0
        hands.append(h)
        ws.append(w.astype(np.float32))
    return hands, ws


def config(name, seed=0, num_hands=None, **over):
    """A seeded subgame description: dict with board, pot, stack, bet_sizes,
    max_raises, num_players, hands, weights and (for non-river) a leaf-value
    generator."""
    rng = np.random.default_rng(seed)
    deck = rng.permutation(52)
    if name == "hu_river":
        board = [int(c) for c in deck[:5]]
        cfg = dict(board=board, pot=100, stack=400, bet_sizes=[0.5, 1.0], max_raises=2,
                   num_players=2, iterations=1000)
        hands, ws = make_ranges(rng, board, 2, num_hands)
    elif name == "turn3":
        board = [int(c) for c in deck[:4]]
        cfg = dict(board=board, pot=150, stack=500, bet_sizes=[0.33, 0.75, 1.5], max_raises=3,
                   num_players=3, iterations=1000, leaf_sigma=0.3 * 150)
        hands, ws = make_ranges(rng, board, 3, num_hands, zero_frac=0.3)
    elif name == "river6":
        board = [int(c) for c in deck[:5]]
        cfg = dict(board=board, pot=300, stack=1000, bet_sizes=[0.5, 1.0], max_raises=2,
                   num_players=6, iterations=2000)
        hands, ws = make_ranges(rng, board, 6, num_hands, weights="dirichlet")
    else:
        raise KeyError(name)
    cfg.update(over)
    cfg["hands"], cfg["weights"], cfg["seed"], cfg["name"] = hands, ws, seed, name
    return cfg


def padded(cfg):
    """hands [np, max_h, 2], weights [np, max_h], num_hands [np]."""
    np_ = cfg["num_players"]
    nh = np.array([len(h) for h in cfg["hands"]], np.int32)
    mh = int(nh.max())
    H = np.zeros((np_, mh, 2), np.int32)
    W = np.zeros((np_, mh), np.float32)
    for p in range(np_):
        H[p, :nh[p]] = cfg["hands"][p]
        W[p, :nh[p]] = cfg["weights"][p]
    return H, W, nh


def leaf_values_for(cfg, num_leaves, seed_offset=1000):
    if num_leaves == 0:
        return None
    rng = np.random.default_rng(cfg["seed"] + seed_offset)
    mh = max(len(h) for h in cfg["hands"])
    return rng.normal(0.0, cfg.get("leaf_sigma", 30.0),
                      (num_leaves, cfg["num_players"], mh)).astype(np.float32)


class AbiSubgame:
    """One subgame driven through the C ABI of libstreet_solve(_wide).so."""

    def __init__(self, cfg, max_hands=None, acting_order=None, use_cont_strats=True):
        need = max(len(h) for h in cfg["hands"])
        self.max_hands_cap = max_hands or (ssg.SS_MAX_HANDS if need <= ssg.SS_MAX_HANDS
                                           else ssg.SS_MAX_HANDS_WIDE)
        self.lib = ssg.load_library(self.max_hands_cap)
        self.cfg = cfg
        np_ = cfg["num_players"]
        order = list(range(np_)) if acting_order is None else acting_order
        board = cfg["board"]
        self.td = ssg.tree_struct(self.max_hands_cap)()
        b = (ctypes.c_int * len(board))(*board)
        s = (ctypes.c_float * len(cfg["bet_sizes"]))(*cfg["bet_sizes"])
        o = (ctypes.c_int * np_)(*order)
        rc = self.lib.ss_build_tree_ex(b, len(board), cfg["pot"], cfg["stack"], s, len(cfg["bet_sizes"]),
                                       np_, o, int(len(board) == 5),
                                       int(use_cont_strats and len(board) < 5), cfg["max_raises"],
                                       ctypes.byref(self.td))
        if rc != 0:
            raise RuntimeError(f"ss_build_tree_ex failed ({rc}): {ssg.last_error(self.lib)}")
        self.H, self.W, self.nh = padded(cfg)
        for p in range(np_):
            self.td.num_hands[p] = int(self.nh[p])
            arr_h = np.ctypeslib.as_array(self.td.hands[p])
            arr_h[:self.nh[p]] = self.H[p, :self.nh[p]]
            arr_w = np.ctypeslib.as_array(self.td.weights[p])
            arr_w[:self.nh[p]] = self.W[p, :self.nh[p]]
        self.leaf_values = None
        self.frozen = None

    @property
    def num_leaves(self):
        return self.td.num_leaves

    def set_leaf_values(self, lv):
        self.leaf_values = None if lv is None else np.ascontiguousarray(lv, np.float32)
        self.td.leaf_values = (None if lv is None else
                               self.leaf_values.ctypes.data_as(ctypes.POINTER(ctypes.c_float)))

    def set_frozen(self, frozen):
        self.frozen = None if frozen is None else np.ascontiguousarray(frozen, np.int32)
        self.td.frozen_action = (None if frozen is None else
                                 self.frozen.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))

    def tree_arrays(self):
        n = self.td.num_nodes
        nodes = np.ctypeslib.as_array(ctypes.cast(self.td.nodes, ctypes.POINTER(ctypes.c_int)),
                                      shape=(n * NODE_INTS,)).reshape(n, NODE_INTS).copy()
        ch = np.ctypeslib.as_array(self.td.children, shape=(max(self.td.num_children_total, 1),))[
            :self.td.num_children_total].copy()
        lo = np.ctypeslib.as_array(self.td.level_order, shape=(n,)).copy()
        nd = np.ctypeslib.as_array(self.td.node_depth, shape=(n,)).copy()
        return nodes, ch, lo, nd

    def solve(self, iterations, graph_iterations=10, device=0, target=None, check_every=50):
        out = ssg.SSOutput()
        stats = ssg.SSSolveStats()
        opts = ssg.SSSolveOptions(device, graph_iterations, -1.0 if target is None else target, check_every, 0)
        rc = self.lib.ss_solve_gpu_ex(ctypes.byref(self.td), iterations, ctypes.byref(opts),
                                      ctypes.byref(out), ctypes.byref(stats))
        if rc != 0:
            return rc, None
        res = read_output(out, self.nh)
        res["stats"] = {k: getattr(stats, k) for k, _ in ssg.SSSolveStats._fields_}
        self.lib.ss_free_output(ctypes.byref(out))
        return 0, res

    def free(self):
        self.td.leaf_values = None
        self.td.frozen_action = None
        self.lib.ss_free_tree(ctypes.byref(self.td))

    def __del__(self):
        try:
            if self.td.nodes:
                self.free()
        except Exception:
            pass


def read_output(out, num_hands):
    mh, na, rp, nd = out.max_hands, out.root_num_actions, out.root_player, out.num_avg_nodes
    nh_root = int(num_hands[rp])
    return {
        "root_strategy": np.ctypeslib.as_array(out.root_strategy, shape=(na * nh_root,)).copy()
        .reshape(na, nh_root),
        "root_ev": np.ctypeslib.as_array(out.root_ev, shape=(out.num_players_out * mh,)).copy()[:mh],
        "avg_strategies": np.ctypeslib.as_array(out.avg_strategies, shape=(nd * ssg.SS_MAX_ACTIONS * mh,))
        .copy().reshape(nd, ssg.SS_MAX_ACTIONS, mh),
        "avg_node_ids": np.ctypeslib.as_array(out.avg_strategy_node_ids, shape=(nd,)).copy(),
        "root_player": rp,
        "root_num_actions": na,
    }


# ---------------------------------------------------------------------------
# batched and served forms through the C ABI
# ---------------------------------------------------------------------------

def batch_solve(subgames, iterations, target=None, check_every=25, graph_iterations=10, device=0):
    """Solve AbiSubgames together (ss_batch_solve); returns (rc, [result dicts])."""
    lib = subgames[0].lib
    n = len(subgames)
    TreeP = ctypes.POINTER(ssg.tree_struct(subgames[0].max_hands_cap))
    trees = (TreeP * n)(*[ctypes.pointer(sg.td) for sg in subgames])
    outs = (ssg.SSOutput * n)()
    stats = (ssg.SSSolveStats * n)()
    opts = ssg.SSSolveOptions(device, graph_iterations, -1.0 if target is None else float(target),
                              check_every, 0)
    lib.ss_batch_solve.restype = ctypes.c_int
    rc = lib.ss_batch_solve(trees, n, iterations, ctypes.byref(opts), outs, stats)
    if rc != 0:
        return rc, None
    res = []
    for i, sg in enumerate(subgames):
        r = read_output(outs[i], sg.nh)
        r["stats"] = {k: getattr(stats[i], k) for k, _ in ssg.SSSolveStats._fields_}
        lib.ss_free_output(ctypes.byref(outs[i]))
        res.append(r)
    return 0, res


class SSServerOptions(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("memory_budget_gb", ctypes.c_double),
                ("block_iterations", ctypes.c_int), ("target_exploitability", ctypes.c_float),
                ("max_iterations", ctypes.c_int), ("graph_iterations", ctypes.c_int)]


class Server:
    """Continuous-batching solve server (ss_server_*)."""

    def __init__(self, lib, **kw):
        self.lib = lib
        opts = SSServerOptions()
        lib.ss_server_default_options(ctypes.byref(opts))
        for k, v in kw.items():
            setattr(opts, k, v)
        self.h = ctypes.c_void_p()
        lib.ss_server_create.restype = ctypes.c_int
        lib.ss_server_submit.restype = ctypes.c_int
        lib.ss_server_poll.restype = ctypes.c_int
        lib.ss_server_wait.restype = ctypes.c_int
        lib.ss_server_destroy.argtypes = [ctypes.c_void_p]
        rc = lib.ss_server_create(ctypes.byref(opts), ctypes.byref(self.h))
        if rc != 0:
            raise RuntimeError(f"ss_server_create failed ({rc}): {ssg.last_error(lib)}")

    def submit(self, sg):
        rid = ctypes.c_longlong()
        rc = self.lib.ss_server_submit(self.h, ctypes.byref(sg.td), ctypes.byref(rid))
        if rc != 0:
            raise RuntimeError(f"ss_server_submit failed ({rc}): {ssg.last_error(self.lib)}")
        return rid.value

    def progress(self, rid):
        """(state, iterations run so far): state 0 queued, 1 in the batch, 2 done."""
        st, it = ctypes.c_int(), ctypes.c_int()
        self.lib.ss_server_progress.restype = ctypes.c_int
        rc = self.lib.ss_server_progress(self.h, ctypes.c_longlong(rid), ctypes.byref(st), ctypes.byref(it))
        if rc != 0:
            raise RuntimeError(f"request {rid} failed ({rc}): {ssg.last_error(self.lib)}")
        return st.value, it.value

    def wait(self, rid, num_hands):
        out, stats, lat = ssg.SSOutput(), ssg.SSSolveStats(), ctypes.c_double()
        rc = self.lib.ss_server_wait(self.h, ctypes.c_longlong(rid), ctypes.byref(out), ctypes.byref(stats),
                                     ctypes.byref(lat))
        if rc != 0:
            raise RuntimeError(f"request {rid} failed ({rc}): {ssg.last_error(self.lib)}")
        r = read_output(out, num_hands)
        r["stats"] = {k: getattr(stats, k) for k, _ in ssg.SSSolveStats._fields_}
        r["latency_ms"] = lat.value
        self.lib.ss_free_output(ctypes.byref(out))
        return r

    def close(self):
        if self.h:
            self.lib.ss_server_destroy(self.h)
            self.h = ctypes.c_void_p()


# ---------------------------------------------------------------------------
# request mix of the batched / served forms
# ---------------------------------------------------------------------------

BET_SETS = [[0.5, 1.0], [0.33, 0.75], [1.0], [0.5], [0.33, 0.75, 1.5], [0.75]]


def mix_config(rng, river=0.8, turn=0.15, river3=0.3):
    """One seeded request of the serving mix: 80% river (2 players, or 3 with
    probability river3), 15% turn (2-3 players, continuation leaves), 5% flop
    (2 players, continuation leaves); all non-board combos with U(0,1)
    weights, a U(0, 0.7) fraction zeroed; random bet set and raise cap (so
    tree sizes spread from tens to thousands of nodes)."""
    u = rng.random()
    street = "river" if u < river else ("turn" if u < river + turn else "flop")
    nb = {"river": 5, "turn": 4, "flop": 3}[street]
    if street == "river":
        np_ = 3 if rng.random() < river3 else 2
    else:
        np_ = 2 if street == "flop" else int(rng.integers(2, 4))
    board = [int(c) for c in rng.permutation(52)[:nb]]
    sizes = BET_SETS[int(rng.integers(len(BET_SETS)))]
    if np_ == 3:
        sizes = sizes[:1]
    raises = int(rng.integers(1, 4)) if street == "river" else int(rng.integers(1, 3))
    pot = int(rng.integers(50, 400))
    cfg = dict(board=board, pot=pot, stack=int(pot * rng.uniform(2, 8)), bet_sizes=sizes,
               max_raises=raises, num_players=np_, seed=int(rng.integers(1 << 30)),
               leaf_sigma=0.3 * pot, name=f"{street}{np_}")
    cfg["hands"], cfg["weights"] = make_ranges(rng, board, np_, None, zero_frac=float(rng.uniform(0, 0.7)))
    return cfg


# ---------------------------------------------------------------------------
# the batched benchmark's request mix: flop / turn / river, 2-6 players, tree
# sizes log-uniform in [50, 20000] nodes, 0-70% of each range zeroed
# ---------------------------------------------------------------------------

SIZE_BETS = [[1.0], [0.75], [0.5], [0.5, 1.0], [0.33, 0.75], [0.33, 0.75, 1.5], [0.25, 0.5, 1.0, 2.0]]
SIZE_RAISES = (1, 2, 3)
# players per street: continuation leaves multiply a leaf by 4^N profiles, so
# flops stay at 2-3 players and turns at 2-4; rivers take 2-6
STREET_PLAYERS = {"flop": (2, 3), "turn": (2, 3, 4), "river": (2, 3, 4, 5, 6)}
_SIZE_TABLE = {}


def _tree_nodes(lib, nb, np_, bets, raises, pot=100, stack=400):
    td = ssg.tree_struct(ssg.SS_MAX_HANDS_WIDE)()
    b = (ctypes.c_int * nb)(*range(0, 4 * nb, 4))
    s = (ctypes.c_float * len(bets))(*bets)
    o = (ctypes.c_int * np_)(*range(np_))
    rc = lib.ss_build_tree_ex(b, nb, pot, stack, s, len(bets), np_, o, int(nb == 5), int(nb < 5), raises,
                              ctypes.byref(td))
    if rc != 0:
        raise RuntimeError(f"ss_build_tree_ex failed ({rc})")
    n = td.num_nodes
    lib.ss_free_tree(ctypes.byref(td))
    return n


def size_table(street, np_):
    """[(nodes, bet_sizes, max_raises)] of every candidate shape (stack = 4 pots)."""
    key = (street, np_)
    if key not in _SIZE_TABLE:
        lib = ssg.load_library(ssg.SS_MAX_HANDS_WIDE)
        nb = {"flop": 3, "turn": 4, "river": 5}[street]
        tab = sorted((_tree_nodes(lib, nb, np_, b, r), b, r) for b in SIZE_BETS for r in SIZE_RAISES)
        if np_ >= 5:
            tab = [e for e in tab if e[0] <= MULTIWAY_MAX_NODES] or tab[:1]
        _SIZE_TABLE[key] = tab
    return _SIZE_TABLE[key]


# 5-6 player trees: at most this many nodes, so that their terminals without
# a closed form (4-5 counted opponents, enumerated) stay within the solver's
# per-solve budget of tuple visits at the ranges below
MULTIWAY_MAX_NODES = 3000


def range_size(np_, rng):
    """Hands per player: every combo for 2-3 players; multiway ranges are
    narrow (4 players 64-128 hands, 5 players 6, 6 players 4), which keeps the
    terminals without a closed form (4-5 counted opponents) enumerable."""
    if np_ <= 3:
        return None
    if np_ == 4:
        return int(rng.integers(64, 129))
    return 6 if np_ == 5 else 4


def c4_config(rng, streets=(1 / 3, 1 / 3, 1 / 3), size=(50, 20000)):
    """One seeded request of the batched mix.  A target size is drawn
    log-uniform in `size`, then a street (weights flop, turn, river) and a
    player count whose trees can come near the target; the bet set and raise
    cap are the candidate shape nearest the target (log scale)."""
    target = float(np.exp(rng.uniform(np.log(size[0]), np.log(size[1]))))
    street = ["flop", "turn", "river"][int(rng.choice(3, p=np.asarray(streets) / np.sum(streets)))]
    cands = []
    for np_ in STREET_PLAYERS[street]:
        tab = size_table(street, np_)
        lo, hi = tab[0][0], tab[-1][0]
        miss = 0.0 if lo <= target <= hi else min(abs(np.log(target / lo)), abs(np.log(target / hi)))
        cands.append((miss, np_))
    best = min(m for m, _ in cands)
    players = [p for m, p in cands if m <= best + 1e-9]
    np_ = int(players[int(rng.integers(len(players)))])
    tab = size_table(street, np_)
    nodes, sizes, raises = min(tab, key=lambda e: abs(np.log(e[0] / target)))
    nb = {"flop": 3, "turn": 4, "river": 5}[street]
    board = [int(c) for c in rng.permutation(52)[:nb]]
    pot = int(rng.integers(50, 400))
    cfg = dict(board=board, pot=pot, stack=4 * pot, bet_sizes=list(sizes), max_raises=int(raises),
               num_players=np_, seed=int(rng.integers(1 << 30)), leaf_sigma=0.3 * pot,
               name=f"{street}{np_}", target_nodes=target)
    cfg["hands"], cfg["weights"] = make_ranges(rng, board, np_, range_size(np_, rng),
                                               zero_frac=float(rng.uniform(0, 0.7)))
    return cfg


def c4_subgames(n, seed=0, streets=(1 / 3, 1 / 3, 1 / 3)):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        cfg = c4_config(rng, streets)
        sg = AbiSubgame(cfg, max_hands=ssg.SS_MAX_HANDS_WIDE)
        sg.set_leaf_values(leaf_values_for(cfg, sg.num_leaves))
        out.append(sg)
    return out


def mix_subgames(n, seed=0):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        cfg = mix_config(rng)
        sg = AbiSubgame(cfg, max_hands=ssg.SS_MAX_HANDS_WIDE)
        sg.set_leaf_values(leaf_values_for(cfg, sg.num_leaves))
        out.append(sg)
    return out
