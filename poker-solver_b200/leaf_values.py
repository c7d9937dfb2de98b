"""Continuation values of depth-limited turn and flop subgames, computed on the GPU.

Host side of the producer the realtime path runs before a turn or flop
solve, with the names, arguments, errors and results of the reference module
python/leaf_values.py:

  compute_turn_leaf_values   python/leaf_values.py:694-816
  compute_flop_leaf_equity   python/leaf_values.py:408-571
  extract_leaf_info_from_tree, LeafInfo   :186-262
  biased_leaf_value, BIAS_FOLD_PROB, BIAS_POT_FACTOR   :84-121

The values are the reference's bit for bit; the computation runs in the
library (ss_leaf_values_gpu, csrc/ss_leaf.cu) and fails with RuntimeError
when it cannot (no library, no CUDA device).  What stays in Python is the
reference's own host logic: the runout draws with numpy's RandomState and
the leaf descriptors read from the tree.  The blueprint-driven producer
(compute_flop_leaf_values) and the strategy-biasing helpers are not part
of this path.  One difference: a range holding more hands than max_hands
raises ValueError up front (the reference fails with an IndexError once
such a hand is live)."""
import ctypes
from collections import namedtuple
from typing import List, Optional, Tuple

import numpy as np

try:
    import street_solver_gpu as ssg
except ImportError:  # imported as part of a package
    from . import street_solver_gpu as ssg

LeafInfo = namedtuple("LeafInfo", ["leaf_idx", "pot", "bets"])

# per continuation profile: 0 unmodified, 1 fold-biased, 2 call-biased, 3 raise-biased
BIAS_FOLD_PROB = [0.0, 0.35, 0.0, 0.0]
BIAS_POT_FACTOR = [1.0, 0.7, 1.0, 1.4]

RUNOUT_SAMPLES = 12      # turn or river cards kept per street when some range is large
LARGE_RANGE = 50         # ... i.e. holds more than this many hands
TUPLE_LIMIT = 2000       # opponent tuples scored per runout and hero player (SS_LEAF_TUPLE_LIMIT)

SS_NODE_DECISION = 0
SS_NODE_LEAF = 4


class SSLeafValueInput(ctypes.Structure):
    """Mirror of SSLeafValueInput (include/street_solve.h)."""
    _fields_ = [
        ("num_players", ctypes.c_int),
        ("max_hands", ctypes.c_int),
        ("num_hands", ctypes.POINTER(ctypes.c_int)),
        ("hand_cards", ctypes.POINTER(ctypes.c_int)),
        ("board", ctypes.POINTER(ctypes.c_int)),
        ("num_board", ctypes.c_int),
        ("runout_cards", ctypes.POINTER(ctypes.c_int)),
        ("num_runouts", ctypes.c_int),
        ("leaf_idx", ctypes.POINTER(ctypes.c_int)),
        ("leaf_pot", ctypes.POINTER(ctypes.c_double)),
        ("num_leaves", ctypes.c_int),
    ]


def _library():
    # the entry point is the same in both builds: reuse one that is loaded already
    lib = ssg.loaded_library() or ssg.load_library()
    if not getattr(lib, "_leaf_bound", False):
        ip = ctypes.POINTER(ctypes.c_int)
        lib.ss_leaf_values_gpu.restype = ctypes.c_int
        lib.ss_leaf_values_gpu.argtypes = [ctypes.POINTER(SSLeafValueInput), ctypes.POINTER(ctypes.c_float)]
        lib.ss_leaf_opponent_tuples.restype = ctypes.c_int
        lib.ss_leaf_opponent_tuples.argtypes = [ctypes.c_int, ip, ip, ctypes.c_int]
        lib._leaf_bound = True
    return lib


def biased_leaf_value(equity, leaf_pot, s_self, s_opp):
    """First-order bias-adjusted value of one hand at one leaf
    (python/leaf_values.py:91-121): with the opponent's fold probability the
    hand collects half the pot, otherwise (equity - 1/2) of the pot scaled by
    both profiles' pot factors."""
    fold = BIAS_FOLD_PROB[s_opp]
    showdown_pot = leaf_pot * (BIAS_POT_FACTOR[s_self] * BIAS_POT_FACTOR[s_opp])
    return fold * (0.5 * leaf_pot) + (1.0 - fold) * ((equity - 0.5) * showdown_pot)


def extract_leaf_info_from_tree(tree_data, num_players=2) -> List[LeafInfo]:
    """Leaf descriptors of a tree from ss_build_tree with continuation leaves
    (python/leaf_values.py:189-262): one per decision node of player 0 that
    heads a full continuation chain -- num_players levels of 4-way decision
    nodes ending in leaf nodes -- with the original leaf index (the first
    chain leaf's leaf_idx // 4^num_players), the node's pot and bets; sorted
    by leaf index."""
    nodes, children = tree_data.nodes, tree_data.children
    per = 4 ** num_players

    def kids(x):
        n = nodes[x]
        return [children[n.first_child + a] for a in range(4)]

    def heads_chain(x):
        frontier = [x]
        for level in range(num_players):
            for y in frontier:
                if nodes[y].type != SS_NODE_DECISION or nodes[y].num_children != 4:
                    return False
            frontier = [z for y in frontier for z in kids(y)]
        return all(nodes[z].type == SS_NODE_LEAF for z in frontier)

    out = []
    for x in range(tree_data.num_nodes):
        n = nodes[x]
        if n.type != SS_NODE_DECISION or n.player != 0 or n.num_children != 4 or not heads_chain(x):
            continue
        y = x
        for _ in range(num_players):
            y = children[nodes[y].first_child]
        out.append(LeafInfo(leaf_idx=nodes[y].leaf_idx // per, pot=n.pot,
                            bets=tuple(n.bets[p] for p in range(num_players))))
    out.sort(key=lambda li: li.leaf_idx)
    return out


def turn_runouts(board_4, num_hands):
    """River cards of a turn subgame in averaging order
    (python/leaf_values.py:754-766): all of them, or 12 drawn with
    RandomState(42), sorted, when some range holds more than 50 hands."""
    on_board = set(int(c) for c in board_4)
    rivers = [c for c in range(52) if c not in on_board]
    if len(rivers) > RUNOUT_SAMPLES and any(n > LARGE_RANGE for n in num_hands):
        rivers = sorted(np.random.RandomState(42).choice(rivers, RUNOUT_SAMPLES, replace=False))
    return [[int(r)] for r in rivers]


def flop_runouts(flop_board, num_hands):
    """(turn, river) cards of a flop subgame in averaging order
    (python/leaf_values.py:479-499): per street all cards, or 12 drawn --
    turns with RandomState(42), the rivers of turn card tc with
    RandomState(43 + tc) -- when some range holds more than 50 hands."""
    on_board = set(int(c) for c in flop_board)
    large = any(n > LARGE_RANGE for n in num_hands)
    turns = [c for c in range(52) if c not in on_board]
    if len(turns) > RUNOUT_SAMPLES and large:
        turns = sorted(np.random.RandomState(42).choice(turns, RUNOUT_SAMPLES, replace=False))
    out = []
    for tc in turns:
        rivers = [c for c in range(52) if c not in on_board and c != tc]
        if len(rivers) > RUNOUT_SAMPLES and large:
            rivers = sorted(np.random.RandomState(43 + int(tc)).choice(rivers, RUNOUT_SAMPLES, replace=False))
        out.extend([int(tc), int(rc)] for rc in rivers)
    return out


def opponent_tuples(list_sizes):
    """The reference's opponent tuples (python/leaf_values.py:615-629) as
    positions into the opponents' live-hand lists, computed by the library's
    host code: int32 [tuples, len(list_sizes)]."""
    lib = _library()
    k = len(list_sizes)
    sizes = np.ascontiguousarray(list_sizes, dtype=np.int32)
    buf = np.zeros((TUPLE_LIMIT, k), dtype=np.int32)
    ip = ctypes.POINTER(ctypes.c_int)
    n = lib.ss_leaf_opponent_tuples(k, sizes.ctypes.data_as(ip), buf.ctypes.data_as(ip), TUPLE_LIMIT)
    if n < 0:
        raise ValueError(f"ss_leaf_opponent_tuples failed ({n}): {ssg.last_error(lib)}")
    return buf[:n].copy()


def _resolve_players(player_hands, oop_hands, ip_hands, who):
    if player_hands is None:
        if oop_hands is None or ip_hands is None:
            raise ValueError(f"{who} requires either player_hands or both oop_hands and ip_hands")
        player_hands = [oop_hands, ip_hands]
    if len(player_hands) < 2 or len(player_hands) > 6:
        raise ValueError(f"{who} supports 2-6 players, got {len(player_hands)}")
    return player_hands


def _produce(board, runouts, leaf_infos, max_hands, player_hands):
    lib = _library()
    N = len(player_hands)
    nh = np.array([len(h) for h in player_hands], dtype=np.int32)
    if int(nh.max()) > max_hands:
        raise ValueError(f"a range holds {int(nh.max())} hands, more than max_hands = {max_hands}")
    cards = np.zeros((N, max(max_hands, 1), 2), dtype=np.int32)
    for p, hands in enumerate(player_hands):
        for h, hand in enumerate(hands):
            cards[p, h, 0], cards[p, h, 1] = int(hand[0]), int(hand[1])
    board_a = np.ascontiguousarray([int(c) for c in board], dtype=np.int32)
    extra = 5 - len(board_a)
    run_a = np.ascontiguousarray(np.array(runouts, dtype=np.int32).reshape(-1, extra))
    idx_a = np.ascontiguousarray([int(li[0]) for li in leaf_infos], dtype=np.int32)
    pot_a = np.ascontiguousarray([float(li[1]) for li in leaf_infos], dtype=np.float64)
    out = np.zeros((len(leaf_infos) * 4 ** N, N, max_hands), dtype=np.float32)
    ip, dp = ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)
    inp = SSLeafValueInput(
        num_players=N, max_hands=max_hands, num_hands=nh.ctypes.data_as(ip), hand_cards=cards.ctypes.data_as(ip),
        board=board_a.ctypes.data_as(ip), num_board=len(board_a), runout_cards=run_a.ctypes.data_as(ip),
        num_runouts=len(run_a), leaf_idx=idx_a.ctypes.data_as(ip), leaf_pot=pot_a.ctypes.data_as(dp),
        num_leaves=len(idx_a))
    rc = lib.ss_leaf_values_gpu(ctypes.byref(inp), out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)))
    if rc != 0:
        raise RuntimeError(f"ss_leaf_values_gpu failed ({rc}): {ssg.last_error(lib)}")
    return out


def compute_turn_leaf_values(
    board_4: List[int],
    leaf_infos: List[LeafInfo],
    max_hands: int,
    starting_pot: int,
    player_hands: Optional[List[List[Tuple[int, int, float]]]] = None,
    oop_hands: Optional[List[Tuple[int, int, float]]] = None,
    ip_hands: Optional[List[Tuple[int, int, float]]] = None,
) -> np.ndarray:
    """Leaf values of a turn subgame for 2-6 players: float32
    [len(leaf_infos) * 4^N, N, max_hands], equity averaged over the river
    cards, bias-adjusted at each leaf's pot.  starting_pot is accepted for
    the reference signature and not used (as there)."""
    player_hands = _resolve_players(player_hands, oop_hands, ip_hands, "compute_turn_leaf_values")
    runouts = turn_runouts(board_4, [len(h) for h in player_hands])
    return _produce(board_4, runouts, leaf_infos, max_hands, player_hands)


def compute_flop_leaf_equity(
    flop_board: List[int],
    leaf_infos: List[LeafInfo],
    max_hands: int,
    starting_pot: int,
    player_hands: Optional[List[List[Tuple[int, int, float]]]] = None,
    oop_hands: Optional[List[Tuple[int, int, float]]] = None,
    ip_hands: Optional[List[Tuple[int, int, float]]] = None,
) -> np.ndarray:
    """Leaf values of a flop subgame for 2-6 players: as
    compute_turn_leaf_values over (turn, river) runouts."""
    player_hands = _resolve_players(player_hands, oop_hands, ip_hands, "compute_flop_leaf_equity")
    runouts = flop_runouts(flop_board, [len(h) for h in player_hands])
    return _produce(flop_board, runouts, leaf_infos, max_hands, player_hands)
