"""Python host side of the B200 street solver.

Drop-in for the reference python/street_solver_gpu.py: the same module name,
struct mirrors (street_solver_gpu.py:66-124), StreetSolverGPU class and
methods (constructor :180-325, set_frozen_actions :327-366, solve :368-373,
get_strategy :375-461, get_avg_strategy :520-548, free :580-596) and the same
action labels (:128-169), bound through ctypes to this repository's
libstreet_solve.so (include/street_solve.h).

Differences a caller can rely on:
  * max_hands=1326 selects libstreet_solve_wide.so, whose SSTreeData holds
    every 2-card combo, so full ranges are solved instead of being trimmed to
    the 200 heaviest hands (street_solver_gpu.py:227-229 trims silently);
  * free() never double-frees leaf values (the reference ss_free_tree frees
    the Python-owned buffer, street_solve.cu:1650);
  * max_raises, solve(..., target_exploitability=...) and exploitability()
    expose the library's extension entry points.
There is no CPU fallback: a missing library raises FileNotFoundError and a
failed call raises RuntimeError with the library's error message.
"""
import ctypes
import os
import sys

import numpy as np

try:
    from cards import card_to_int, int_to_card, parse_range_string  # noqa: F401
except ImportError:  # imported as part of a package
    from .cards import card_to_int, int_to_card, parse_range_string  # noqa: F401

SS_MAX_PLAYERS = 6
SS_MAX_HANDS = 200
SS_MAX_HANDS_WIDE = 1326
SS_MAX_ACTIONS = 8
SS_MAX_BOARD = 5
SS_MAX_RAISES = 3
SCALE = 100

NODE_DECISION, NODE_FOLD, NODE_SHOWDOWN, NODE_LEAF = 0, 1, 2, 4

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_DIR = os.path.join(_PKG, "lib")
_LIB_NAMES = {SS_MAX_HANDS: "libstreet_solve.so", SS_MAX_HANDS_WIDE: "libstreet_solve_wide.so"}
_LIBS = {}
_STRUCTS = {}


class SSNode(ctypes.Structure):
    _fields_ = [
        ("type", ctypes.c_int),
        ("player", ctypes.c_int),
        ("num_children", ctypes.c_int),
        ("first_child", ctypes.c_int),
        ("pot", ctypes.c_int),
        ("bets", ctypes.c_int * SS_MAX_PLAYERS),
        ("board_cards", ctypes.c_int * 5),
        ("num_board", ctypes.c_int),
        ("leaf_idx", ctypes.c_int),
        ("fold_player", ctypes.c_int),
        ("num_players", ctypes.c_int),
        ("active_players", ctypes.c_int * SS_MAX_PLAYERS),
    ]


class SSOutput(ctypes.Structure):
    _fields_ = [
        ("root_strategy", ctypes.POINTER(ctypes.c_float)),
        ("root_num_actions", ctypes.c_int),
        ("root_player", ctypes.c_int),
        ("root_ev", ctypes.POINTER(ctypes.c_float)),
        ("avg_strategies", ctypes.POINTER(ctypes.c_float)),
        ("avg_strategy_node_ids", ctypes.POINTER(ctypes.c_int)),
        ("num_avg_nodes", ctypes.c_int),
        ("num_players_out", ctypes.c_int),
        ("max_hands", ctypes.c_int),
    ]


class SSAbiInfo(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in ("abi_version", "max_hands", "max_players",
                                            "max_actions", "sizeof_node", "sizeof_tree",
                                            "sizeof_output")]


class SSSolveOptions(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("graph_iterations", ctypes.c_int),
                ("target_exploitability", ctypes.c_float), ("check_every", ctypes.c_int),
                ("compute_exploitability", ctypes.c_int)]


class SSSolveStats(ctypes.Structure):
    _fields_ = [("iterations_run", ctypes.c_int), ("exploitability_pct", ctypes.c_double),
                ("nashconv", ctypes.c_double), ("solve_ms", ctypes.c_double),
                ("node_hand_updates", ctypes.c_double), ("queue_ms", ctypes.c_double)]


def tree_struct(max_hands=SS_MAX_HANDS):
    """ctypes mirror of SSTreeData for a given SS_MAX_HANDS."""
    if max_hands in _STRUCTS:
        return _STRUCTS[max_hands]

    class SSTreeData(ctypes.Structure):
        _fields_ = [
            ("nodes", ctypes.POINTER(SSNode)),
            ("children", ctypes.POINTER(ctypes.c_int)),
            ("num_nodes", ctypes.c_int),
            ("num_children_total", ctypes.c_int),
            ("num_players_field", ctypes.c_int),
            ("hands", ((ctypes.c_int * 2) * max_hands) * SS_MAX_PLAYERS),
            ("weights", (ctypes.c_float * max_hands) * SS_MAX_PLAYERS),
            ("num_hands", ctypes.c_int * SS_MAX_PLAYERS),
            ("board", ctypes.c_int * SS_MAX_BOARD),
            ("num_board", ctypes.c_int),
            ("leaf_values", ctypes.POINTER(ctypes.c_float)),
            ("num_leaves", ctypes.c_int),
            ("level_order", ctypes.POINTER(ctypes.c_int)),
            ("node_depth", ctypes.POINTER(ctypes.c_int)),
            ("max_depth", ctypes.c_int),
            ("decision_node_indices", ctypes.POINTER(ctypes.c_int)),
            ("num_decision_nodes", ctypes.c_int),
            ("showdown_node_indices", ctypes.POINTER(ctypes.c_int)),
            ("num_showdown_nodes", ctypes.c_int),
            ("leaf_node_indices", ctypes.POINTER(ctypes.c_int)),
            ("num_leaf_nodes", ctypes.c_int),
            ("fold_node_indices", ctypes.POINTER(ctypes.c_int)),
            ("num_fold_nodes", ctypes.c_int),
            ("starting_pot", ctypes.c_int),
            ("effective_stack", ctypes.c_int),
            ("is_river", ctypes.c_int),
            ("frozen_action", ctypes.POINTER(ctypes.c_int)),
        ]

    _STRUCTS[max_hands] = SSTreeData
    return SSTreeData


SSTreeData = tree_struct(SS_MAX_HANDS)


def library_path(max_hands=SS_MAX_HANDS):
    return os.path.join(LIB_DIR, _LIB_NAMES[max_hands])


def load_library(max_hands=SS_MAX_HANDS):
    """Load (once) the library build for max_hands (200 or 1326)."""
    if max_hands in _LIBS:
        return _LIBS[max_hands]
    if max_hands not in _LIB_NAMES:
        raise ValueError("max_hands must be 200 or 1326")
    path = library_path(max_hands)
    if not os.path.exists(path):
        raise FileNotFoundError(
            f"street solver library not found at {path}; build it with "
            f"'python poker-solver_b200/build.py'")
    lib = ctypes.CDLL(path)
    T = ctypes.POINTER(tree_struct(max_hands))
    fp, ip = ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_int)
    lib.ss_build_tree.restype = ctypes.c_int
    lib.ss_build_tree_ex.restype = ctypes.c_int
    lib.ss_build_tree_ex.argtypes = [ip, ctypes.c_int, ctypes.c_int, ctypes.c_int, fp, ctypes.c_int,
                                     ctypes.c_int, ip, ctypes.c_int, ctypes.c_int, ctypes.c_int, T]
    lib.ss_solve_gpu.restype = ctypes.c_int
    lib.ss_solve_gpu_ex.restype = ctypes.c_int
    lib.ss_solve_gpu_ex.argtypes = [T, ctypes.c_int, ctypes.POINTER(SSSolveOptions),
                                    ctypes.POINTER(SSOutput), ctypes.POINTER(SSSolveStats)]
    lib.ss_free_tree.restype = None
    lib.ss_free_output.restype = None
    lib.ss_abi_info.restype = ctypes.c_int
    lib.ss_last_error.restype = ctypes.c_char_p
    lib.ss_exploitability_gpu.restype = ctypes.c_int
    dp = ctypes.POINTER(ctypes.c_double)
    lib.ss_exploitability_gpu.argtypes = [T, fp, dp, dp, dp, dp, dp]
    info = SSAbiInfo()
    lib.ss_abi_info(ctypes.byref(info))
    if (info.max_hands != max_hands or info.sizeof_tree != ctypes.sizeof(tree_struct(max_hands))
            or info.sizeof_node != ctypes.sizeof(SSNode)
            or info.sizeof_output != ctypes.sizeof(SSOutput)):
        raise RuntimeError(f"ABI mismatch between {path} and the Python mirrors")
    _LIBS[max_hands] = lib
    return lib


def _session_api(lib):
    """ctypes signatures of the resident-session entry points."""
    vp = ctypes.c_void_p
    lib.ss_session_create.restype = ctypes.c_int
    lib.ss_session_run.restype = ctypes.c_int
    lib.ss_session_run.argtypes = [vp, ctypes.c_int]
    lib.ss_session_output.restype = ctypes.c_int
    lib.ss_session_output.argtypes = [vp, ctypes.POINTER(SSOutput)]
    lib.ss_session_destroy.restype = None
    lib.ss_session_destroy.argtypes = [vp]
    lib.ss_session_narrow.restype = ctypes.c_int
    lib.ss_session_narrow.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_uint, ctypes.c_int,
                                      ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double),
                                      ctypes.POINTER(ctypes.c_int)]


def loaded_library():
    """A library build already loaded in this process (either layout), or
    None -- for entry points that do not depend on SS_MAX_HANDS."""
    return next(iter(_LIBS.values()), None)


def last_error(lib):
    msg = lib.ss_last_error()
    return msg.decode() if msg else ""


# ── Action labels (reference street_solver_gpu.py:128-169) ───────────────

def _build_labels_at_node(tree_data, node_idx):
    """Labels of a decision node's actions: Fold, Check / Call, Bet x% / Raise x%
    with x the actor's bet increase as a percentage of the node's pot."""
    node = tree_data.nodes[node_idx]
    actor = node.player
    own = node.bets[actor] if actor >= 0 else 0
    top = max(node.bets[p] for p in range(SS_MAX_PLAYERS))
    to_call = top - own if actor >= 0 else 0
    labels = []
    for i in range(node.num_children):
        child = tree_data.nodes[tree_data.children[node.first_child + i]]
        if child.type == NODE_FOLD:
            labels.append("Fold")
        elif child.type in (NODE_SHOWDOWN, NODE_LEAF):
            labels.append("Call" if to_call > 0 else "Check")
        elif child.type == NODE_DECISION:
            amount = (child.bets[actor] if actor >= 0 else 0) - own
            if amount == 0:
                labels.append("Check")
            elif node.pot > 0:
                pct = int(round(100 * amount / node.pot))
                labels.append(f"Raise {pct}%" if to_call > 0 else f"Bet {pct}%")
            else:
                labels.append("Bet" if to_call == 0 else "Raise")
        else:
            labels.append(f"Action {i}")
    return labels


class StreetSolverGPU:
    """N-player single-street Linear-CFR solver on one B200.

    Same constructor and methods as the reference class; see the module
    docstring for the additions."""

    def __init__(self, board, pot_bb, stack_bb,
                 oop_range=None, ip_range=None,
                 player_ranges=None,
                 acting_order=None,
                 bet_sizes=None, leaf_values=None,
                 use_cont_strats=True, leaf_value_fn=None,
                 max_hands=None, max_raises=SS_MAX_RAISES):
        self._freed = True
        self.max_hands_cap = SS_MAX_HANDS if max_hands is None else int(max_hands)
        self.lib = load_library(self.max_hands_cap)

        self.board_cards = [card_to_int(c) for c in board] if isinstance(board[0], str) else list(board)
        self.num_board = len(self.board_cards)
        self.is_river = self.num_board == 5
        board_set = set(self.board_cards)

        if player_ranges is not None:
            ranges = list(player_ranges)
        elif oop_range is not None and ip_range is not None:
            ranges = [oop_range, ip_range]
        else:
            raise ValueError("Provide oop_range+ip_range or player_ranges")
        self.num_players = len(ranges)
        self.player_hands = []
        for r in ranges:
            hands = parse_range_string(r) if isinstance(r, str) else list(r)
            hands = [(c0, c1, w) for c0, c1, w in hands if c0 not in board_set and c1 not in board_set]
            if len(hands) > self.max_hands_cap:
                hands.sort(key=lambda x: -x[2])
                hands = hands[:self.max_hands_cap]
            self.player_hands.append(hands)
        self.oop_hands = self.player_hands[0]
        if self.num_players >= 2:
            self.ip_hands = self.player_hands[1]

        self.bet_sizes = [0.33, 0.75, 1.5] if bet_sizes is None else bet_sizes
        self.acting_order = list(range(self.num_players)) if acting_order is None else acting_order
        pot = int(pot_bb * SCALE)
        stack = int(stack_bb * SCALE)

        Tree = tree_struct(self.max_hands_cap)
        self._tree = Tree()
        b = (ctypes.c_int * self.num_board)(*self.board_cards)
        s = (ctypes.c_float * len(self.bet_sizes))(*self.bet_sizes)
        o = (ctypes.c_int * len(self.acting_order))(*self.acting_order)
        err = self.lib.ss_build_tree_ex(b, self.num_board, pot, stack, s, len(self.bet_sizes),
                                        self.num_players, o, 1 if self.is_river else 0,
                                        1 if (use_cont_strats and not self.is_river) else 0,
                                        int(max_raises), ctypes.byref(self._tree))
        if err != 0:
            raise RuntimeError(f"ss_build_tree failed ({err}): {last_error(self.lib)}")
        self._freed = False

        for p in range(self.num_players):
            self._tree.num_hands[p] = len(self.player_hands[p])
            for i, (c0, c1, w) in enumerate(self.player_hands[p]):
                self._tree.hands[p][i][0] = c0
                self._tree.hands[p][i][1] = c1
                self._tree.weights[p][i] = w
        self._max_hands = max(len(h) for h in self.player_hands)

        if leaf_values is None and leaf_value_fn is not None and self._tree.num_leaves > 0:
            leaf_values = leaf_value_fn(self._tree, self.player_hands, self._max_hands,
                                        int(pot_bb * SCALE))
        self._leaf_arr = None
        if leaf_values is not None and self._tree.num_leaves > 0:
            expected = self._tree.num_leaves * self.num_players * self._max_hands
            flat = np.ascontiguousarray(np.asarray(leaf_values, dtype=np.float32).ravel())
            if flat.size != expected:
                raise ValueError(
                    f"leaf_values mismatch: {flat.size} vs {expected} (leaves={self._tree.num_leaves}, "
                    f"players={self.num_players}, max_hands={self._max_hands})")
            self._leaf_arr = flat
            self._tree.leaf_values = flat.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
        elif not self.is_river and self._tree.num_leaves > 0:
            print("[WARNING] Zero leaf values — no blueprint data.", file=sys.stderr)
            self._leaf_arr = np.zeros(self._tree.num_leaves * self.num_players * self._max_hands,
                                      np.float32)
            self._tree.leaf_values = self._leaf_arr.ctypes.data_as(ctypes.POINTER(ctypes.c_float))

        self._frozen_arr = None
        self._output = SSOutput()
        self._solved = False
        self.stats = None

    # ── freezing (reference street_solver_gpu.py:327-366) ───────────────
    def set_frozen_actions(self, frozen_actions, hero_player):
        """Walk the tree along the given action labels (any player's) and
        freeze hero's nodes on the action taken."""
        n = self._tree.num_nodes
        frozen = (ctypes.c_int * n)(*([-1] * n))
        cur = 0
        for label in frozen_actions:
            node = self._tree.nodes[cur]
            if node.type != NODE_DECISION:
                break
            labels = _build_labels_at_node(self._tree, cur)
            hit = next((i for i, lb in enumerate(labels) if lb.lower() == label.lower()), -1)
            if hit < 0:
                break
            if node.player == hero_player:
                frozen[cur] = hit
            cur = self._tree.children[node.first_child + hit]
        self._frozen_arr = frozen
        self._tree.frozen_action = ctypes.cast(frozen, ctypes.POINTER(ctypes.c_int))

    # ── solving ──────────────────────────────────────────────────────────
    def solve(self, iterations=200, target_exploitability=None, graph_iterations=10, device=0,
              compute_exploitability=False, resident=False):
        """resident=True keeps the solve's state on the GPU as a session (for
        narrow_weights, more iterations, reads); otherwise one ss_solve_gpu_ex
        call that allocates and releases everything."""
        if self._solved:
            self.lib.ss_free_output(ctypes.byref(self._output))
            self._solved = False
        opts = SSSolveOptions(device, graph_iterations,
                              -1.0 if target_exploitability is None else float(target_exploitability),
                              50, 1 if compute_exploitability else 0)
        stats = SSSolveStats()
        if resident:
            self._drop_session()
            _session_api(self.lib)
            sess = ctypes.c_void_p()
            err = self.lib.ss_session_create(ctypes.byref(self._tree), ctypes.byref(opts), ctypes.byref(sess))
            if err != 0:
                raise RuntimeError(f"ss_session_create failed ({err}): {last_error(self.lib)}")
            self._session = sess
            err = self.lib.ss_session_run(sess, int(iterations))
            if err == 0:
                err = self.lib.ss_session_output(sess, ctypes.byref(self._output))
            if err != 0:
                raise RuntimeError(f"session solve failed ({err}): {last_error(self.lib)}")
            stats.iterations_run = int(iterations)
            stats.exploitability_pct = -1.0
            self._solved = True
            self.stats = stats
            return stats
        err = self.lib.ss_solve_gpu_ex(ctypes.byref(self._tree), int(iterations), ctypes.byref(opts),
                                       ctypes.byref(self._output), ctypes.byref(stats))
        if err != 0:
            raise RuntimeError(f"ss_solve_gpu failed ({err}): {last_error(self.lib)}")
        self._solved = True
        self.stats = stats
        return stats

    def exploitability(self):
        """FP64 exploitability of the current average strategy, % of pot."""
        if not self._solved:
            raise RuntimeError("Must call solve() first")
        pct, nc = ctypes.c_double(), ctypes.c_double()
        br = (ctypes.c_double * SS_MAX_PLAYERS)()
        cur = (ctypes.c_double * SS_MAX_PLAYERS)()
        z = ctypes.c_double()
        err = self.lib.ss_exploitability_gpu(ctypes.byref(self._tree), self._output.avg_strategies,
                                             ctypes.byref(pct), ctypes.byref(nc), br, cur,
                                             ctypes.byref(z))
        if err != 0:
            raise RuntimeError(f"ss_exploitability_gpu failed ({err}): {last_error(self.lib)}")
        return {"exploitability_pct": pct.value, "nashconv": nc.value,
                "br_value": list(br)[:self.num_players], "cur_value": list(cur)[:self.num_players],
                "deal_mass": z.value}

    # ── raw outputs (numpy views copied out) ─────────────────────────────
    def avg_strategies_array(self):
        o = self._output
        n = o.num_avg_nodes * SS_MAX_ACTIONS * o.max_hands
        return np.ctypeslib.as_array(o.avg_strategies, shape=(n,)).copy().reshape(
            o.num_avg_nodes, SS_MAX_ACTIONS, o.max_hands)

    def root_strategy_array(self):
        o = self._output
        nh = len(self.player_hands[o.root_player])
        return np.ctypeslib.as_array(o.root_strategy, shape=(o.root_num_actions * nh,)).copy().reshape(
            o.root_num_actions, nh)

    def root_ev_array(self):
        o = self._output
        return np.ctypeslib.as_array(o.root_ev, shape=(o.num_players_out * o.max_hands,)).copy()[:o.max_hands]

    # ── strategy queries (reference street_solver_gpu.py:375-548) ──────
    def get_strategy(self, player, hand_str=None, hand_idx=None, frozen_actions=None):
        if not self._solved:
            raise RuntimeError("Must call solve() first")
        pi = self._resolve_player(player)
        if hand_idx is None:
            hand_idx = self._find_hand(pi, hand_str)
        if not frozen_actions:
            if self._output.root_player == pi:
                nh = len(self.player_hands[pi])
                labels = _build_labels_at_node(self._tree, 0)
                out = {}
                for a in range(min(self._output.root_num_actions, len(labels))):
                    f = self._output.root_strategy[a * nh + hand_idx]
                    if f > 0.001:
                        out[labels[a]] = float(f)
                return out
            return self._get_strategy_at_player_node(pi, hand_idx)
        cur, k = 0, 0
        while k < len(frozen_actions) and cur < self._tree.num_nodes:
            node = self._tree.nodes[cur]
            if node.type != NODE_DECISION:
                break
            labels = _build_labels_at_node(self._tree, cur)
            nxt = None
            for ci in range(node.num_children):
                if ci < len(labels) and self._match_action_label(labels[ci], frozen_actions[k]):
                    nxt = self._tree.children[node.first_child + ci]
                    break
            if nxt is None:
                break
            cur, k = nxt, k + 1
        node = self._tree.nodes[cur]
        if node.type == NODE_DECISION and node.player == pi:
            return self._get_strategy_at_node(cur, pi, hand_idx)
        return self._get_strategy_at_player_node(pi, hand_idx)

    @staticmethod
    def _match_action_label(tree_label, frozen_label):
        return tree_label.lower().strip() == frozen_label.lower().strip()

    def _strategy_row(self, di, nidx, hand_idx):
        node = self._tree.nodes[nidx]
        labels = _build_labels_at_node(self._tree, nidx)
        mh = self._max_hands
        out = {}
        for a in range(min(node.num_children, len(labels))):
            f = self._output.avg_strategies[di * SS_MAX_ACTIONS * mh + a * mh + hand_idx]
            if f > 0.001:
                out[labels[a]] = float(f)
        return out

    def _get_strategy_at_node(self, node_idx, player_idx, hand_idx):
        for di in range(self._output.num_avg_nodes):
            nidx = self._output.avg_strategy_node_ids[di]
            if nidx != node_idx:
                continue
            node = self._tree.nodes[nidx]
            if node.player != player_idx or node.type != NODE_DECISION:
                continue
            return self._strategy_row(di, nidx, hand_idx)
        return {}

    def _get_strategy_at_player_node(self, player_idx, hand_idx):
        for di in range(self._output.num_avg_nodes):
            nidx = self._output.avg_strategy_node_ids[di]
            node = self._tree.nodes[nidx]
            if node.player != player_idx or node.type != NODE_DECISION:
                continue
            return self._strategy_row(di, nidx, hand_idx)
        return {}

    def get_all_strategies(self, player):
        if not self._solved:
            raise RuntimeError("Must call solve() first")
        pi = self._resolve_player(player)
        out = {}
        for h in range(len(self.player_hands[pi])):
            s = self.get_strategy(pi, hand_idx=h)
            if s:
                out[h] = s
        return out

    def get_avg_strategy(self, player):
        if not self._solved:
            raise RuntimeError("Must call solve() first")
        pi = self._resolve_player(player)
        for di in range(self._output.num_avg_nodes):
            nidx = self._output.avg_strategy_node_ids[di]
            node = self._tree.nodes[nidx]
            if node.type != NODE_DECISION or node.player != pi:
                continue
            out = {}
            for h, (c0, c1, _w) in enumerate(self.player_hands[pi]):
                out[(min(c0, c1), max(c0, c1))] = self._strategy_row(di, nidx, h)
            return out
        return {}

    def get_avg_strategy_probs(self, player, action_label):
        return {k: v.get(action_label, 0.0) for k, v in self.get_avg_strategy(player).items()}

    def _resolve_player(self, player):
        if isinstance(player, int):
            return player
        return {"oop": 0, "ip": 1}.get(player, None) if player in ("oop", "ip") else int(player)

    def _find_hand(self, player_idx, hand_str):
        key = tuple(sorted((card_to_int(hand_str[:2]), card_to_int(hand_str[2:]))))
        for i, (h0, h1, _w) in enumerate(self.player_hands[player_idx]):
            if tuple(sorted((h0, h1))) == key:
                return i
        raise ValueError(f"Hand {hand_str} not in player {player_idx}'s range")

    def narrow_weights(self, player, action_label, hand_cards, weights, node=None):
        """The reference's between-street range update (python/hud_solver.py:
        345-362 with python/range_narrowing.py:83-130) on the GPU from this
        resident solve: P(action_label | hand) from `player`'s average strategy
        at its first decision node (or `node`), applied to the entries
        (hand_cards[i], weights[i]).  Returns (applied, new weights)."""
        if getattr(self, "_session", None) is None:
            raise RuntimeError("narrow_weights needs solve(..., resident=True)")
        pi = self._resolve_player(player)
        nidx = node
        if nidx is None:
            nidx = next((int(self._output.avg_strategy_node_ids[di]) for di in range(self._output.num_avg_nodes)
                         if self._tree.nodes[self._output.avg_strategy_node_ids[di]].player == pi), -1)
        if nidx < 0:
            return False, list(weights)
        labels = _build_labels_at_node(self._tree, nidx)
        mask = sum(1 << a for a, lbl in enumerate(labels) if lbl == action_label)
        if mask == 0:
            return False, list(weights)
        n = len(hand_cards)
        cards = (ctypes.c_int * max(2 * n, 1))(*[c for hc in hand_cards for c in hc])
        w = (ctypes.c_double * max(n, 1))(*weights)
        applied = ctypes.c_int()
        err = self.lib.ss_session_narrow(self._session, pi, nidx, mask, n, cards, w, ctypes.byref(applied))
        if err != 0:
            raise RuntimeError(f"ss_session_narrow failed ({err}): {last_error(self.lib)}")
        return bool(applied.value), list(w)[:n]

    def _drop_session(self):
        if getattr(self, "_session", None) is not None:
            self.lib.ss_session_destroy(self._session)
            self._session = None

    def free(self):
        if getattr(self, "_freed", True):
            return
        self._freed = True
        self._drop_session()
        if getattr(self, "_solved", False):
            self.lib.ss_free_output(ctypes.byref(self._output))
            self._solved = False
        self.lib.ss_free_tree(ctypes.byref(self._tree))

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass
