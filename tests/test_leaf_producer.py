"""Host-side checks of the GPU continuation-value producer
(ss_leaf_values_gpu: poker-solver_b200/leaf_values.py, csrc/ss_leaf*):
* the library's opponent-tuple rule is the reference's -- itertools.product
  up to 2000 tuples, else 2000 drawn with random.Random(42).choice per
  opponent (python/leaf_values.py:615-629) -- for sizes that enumerate and
  sizes that sample;
* the host module draws the reference's runouts and reads its leaf
  descriptors (against the oracle and the reference-generated fixtures);
* the kernels' per-element functions, compiled for the host with g++ into
  tests/native/leaf_emul and run phase by phase over the library's plan,
  reproduce the reference module's leaf values bit for bit
  (tests/golden/leaf_values_*.npz), the oracle's on edge cases (an empty
  range, a range the board blocks entirely, no runouts), and the oracle's
  numpy form at size (a 3-player turn with 1128 hands, six players with
  sampled 5-tuples, a 3-player flop with every runout);
* the leaf descriptors of a 4-player tree match the oracle's walk;
* malformed inputs are refused before any CUDA call, and a valid call on a
  machine without a GPU raises instead of falling back to the CPU."""
import glob
import itertools
import math
import os
import random
import shutil
import subprocess

import numpy as np
import pytest

import leaf_values as lv
import workloads as wl
from conftest import HAVE_GPU
from oracle import leaf_oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "poker-solver_b200", "csrc")
HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "leaf_values_*.npz")))
IDS = [os.path.basename(p)[12:-4] for p in FIXTURES]


def reference_tuples(sizes):
    """python/leaf_values.py:603-629 over lists 0..n-1 (positions)."""
    lists = [list(range(n)) for n in sizes]
    total = math.prod(sizes)
    if total == 0:
        return []
    if total <= 2000:
        return list(itertools.product(*lists))
    rng = random.Random(42)
    return [tuple(rng.choice(lst) for lst in lists) for _ in range(2000)]


@pytest.mark.parametrize("sizes", [(30,), (1081,), (1326,), (0, 5), (10, 10), (44, 45), (45, 45), (52, 52),
                                   (1128, 1128), (7, 9, 11), (12, 13, 14), (2, 1000), (2, 1001), (1, 1),
                                   (40, 41, 42, 43, 44), (1081, 1081, 1081, 1081, 1081)])
def test_tuple_rule_is_the_reference_rule(sizes):
    got = lv.opponent_tuples(list(sizes))
    want = np.array(reference_tuples(sizes), dtype=np.int32).reshape(-1, len(sizes))
    assert got.shape == want.shape
    assert np.array_equal(got, want)


def load_case(path):
    g = np.load(path)
    np_ = int(g["num_players"])
    board = [int(c) for c in g["board"]]
    hands = [g["hands"][p] for p in range(np_)]
    ws = [g["weights"][p] for p in range(np_)]
    ph = [[(int(h[0]), int(h[1]), float(w)) for h, w in zip(hands[p], ws[p])] for p in range(np_)]
    infos = list(zip(g["leaf_idx"].tolist(), g["leaf_pot"].tolist()))
    return g, board, hands, ws, ph, infos


def runouts_for(board, ph):
    nh = [len(h) for h in ph]
    return lv.turn_runouts(board, nh) if len(board) == 4 else lv.flop_runouts(board, nh)


@pytest.mark.parametrize("path", FIXTURES, ids=IDS)
def test_host_runouts_and_descriptors(path):
    g, board, hands, ws, ph, _ = load_case(path)
    ora = (leaf_oracle.turn_runouts if len(board) == 4 else leaf_oracle.flop_runouts)(board, ph)
    assert runouts_for(board, ph) == ora
    cfg = dict(board=board, pot=int(g["pot"]), stack=int(g["stack"]), bet_sizes=[float(x) for x in g["bet_sizes"]],
               max_raises=int(g["max_raises"]), num_players=len(ph), hands=hands, weights=ws)
    sg = wl.AbiSubgame(cfg)
    try:
        infos = lv.extract_leaf_info_from_tree(sg.td, len(ph))
    finally:
        sg.free()
    assert [i.leaf_idx for i in infos] == g["leaf_idx"].tolist()
    assert [i.pot for i in infos] == g["leaf_pot"].tolist()
    assert [list(i.bets) for i in infos] == g["leaf_bets"].tolist()


@pytest.fixture(scope="module")
def emul(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    out = str(tmp_path_factory.mktemp("leaf") / "leaf_emul")
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-I", os.path.join(ROOT, "include"),
                    "-I", CSRC, os.path.join(HERE, "native", "leaf_emul.cpp"),
                    os.path.join(CSRC, "ss_leaf_plan.cpp"), "-o", out], check=True)
    return out


def emulate(driver, tmp_path, board, runouts, infos, max_hands, ph, chunk_rows=None):
    N = len(ph)
    cards = np.zeros((N, max_hands, 2), np.int64)
    for p, hs in enumerate(ph):
        for h, hand in enumerate(hs):
            cards[p, h] = hand[0], hand[1]
    flat_runs = [c for r in runouts for c in r]
    lines = [f"{N} {max_hands} {len(board)} {len(runouts)} {len(infos)}",
             " ".join(str(len(h)) for h in ph), " ".join(map(str, cards.ravel().tolist())),
             " ".join(map(str, board)), " ".join(map(str, flat_runs)),
             " ".join(str(int(i[0])) for i in infos), " ".join(repr(float(i[1])) for i in infos)]
    inp, outp = tmp_path / "in.txt", tmp_path / "out.f32"
    inp.write_text("\n".join(lines) + "\n")
    subprocess.run([driver, str(inp), str(outp)] + ([str(chunk_rows)] if chunk_rows else []), check=True)
    return np.fromfile(outp, np.float32).reshape(len(infos) * 4 ** N, N, max_hands)


@pytest.mark.parametrize("path", FIXTURES, ids=IDS)
def test_element_functions_reproduce_reference_values(emul, tmp_path, path):
    g, board, _, _, ph, infos = load_case(path)
    got = emulate(emul, tmp_path, board, runouts_for(board, ph), infos, int(g["max_hands"]), ph)
    assert got.shape == g["leaf_values"].shape
    assert np.array_equal(got, g["leaf_values"])
    # the value phase in chunks of 7 rows (a tail chunk, rows starting mid-leaf)
    chunked = emulate(emul, tmp_path, board, runouts_for(board, ph), infos, int(g["max_hands"]), ph, chunk_rows=7)
    assert np.array_equal(chunked, g["leaf_values"])


def edge_cases():
    rng = np.random.default_rng(11)
    board = [int(c) for c in rng.permutation(52)[:4]]
    combos = wl.all_combos(board)
    pick = lambda n: [(a, b, 1.0) for a, b in (combos[i] for i in sorted(rng.choice(len(combos), n, replace=False)))]
    blocked = [(board[0], c, 1.0) for c in range(52) if c not in board][:6]   # every hand holds a board card
    infos = [(0, 90), (1, 150), (2, 240)]
    return [
        ("empty_range", board, [pick(9), []], infos, 9),
        ("three_with_empty", board, [pick(6), [], pick(7)], infos[:2], 8),
        ("blocked_range", board, [pick(8), blocked], infos, 8),
        ("four_players", board, [pick(4), pick(3), pick(4), pick(3)], [(0, 200)], 5),
    ]


@pytest.mark.parametrize("case", edge_cases(), ids=lambda c: c[0])
def test_element_functions_on_edge_cases(emul, tmp_path, case):
    _, board, ph, infos, mh = case
    runs = runouts_for(board, ph)
    got = emulate(emul, tmp_path, board, runs, infos, mh, ph)
    want = leaf_oracle.turn_leaf_values(board, [(i, p, ()) for i, p in infos], mh, ph)
    assert np.array_equal(got, want)
    # no runouts: every equity is 0 and the values are the bias terms alone
    got0 = emulate(emul, tmp_path, board, [], infos, mh, ph)
    want0 = leaf_oracle._leaf_values(board, [], [(i, p, ()) for i, p in infos], mh, ph, None)
    assert np.array_equal(got0, want0)


def call_raw(board, runouts, infos, max_hands, ph, num_players=None):
    """ss_leaf_values_gpu through ctypes with a hand-made input; returns (rc, message)."""
    lib = lv._library()
    import ctypes
    N = num_players if num_players is not None else len(ph)
    nh = np.array([len(h) for h in ph] + [0] * max(0, N - len(ph)), np.int32)
    rows = max([max_hands] + [len(h) for h in ph])   # room for a range larger than max_hands (refused)
    cards = np.zeros((max(N, 1), rows, 2), np.int32)
    for p, hs in enumerate(ph):
        for h, hand in enumerate(hs):
            cards[p, h] = hand[0], hand[1]
    b = np.array(board, np.int32)
    r = np.array(runouts, np.int32).reshape(-1, 5 - len(board)) if len(board) in (3, 4) else np.zeros((0, 1), np.int32)
    li = np.array([i for i, _ in infos], np.int32)
    lp = np.array([p for _, p in infos], np.float64)
    out = np.zeros(max(1, len(infos) * 4 ** min(N, 6) * N * max_hands), np.float32)
    ip, dp = ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)
    inp = lv.SSLeafValueInput(num_players=N, max_hands=max_hands, num_hands=nh.ctypes.data_as(ip),
                              hand_cards=cards.ctypes.data_as(ip), board=b.ctypes.data_as(ip), num_board=len(b),
                              runout_cards=r.ctypes.data_as(ip), num_runouts=len(r),
                              leaf_idx=li.ctypes.data_as(ip), leaf_pot=lp.ctypes.data_as(dp), num_leaves=len(li))
    rc = lib.ss_leaf_values_gpu(ctypes.byref(inp), out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)))
    return rc, lv.ssg.last_error(lib)


def test_malformed_inputs_are_refused():
    board = [0, 5, 10, 15]
    ph = [[(20, 21, 1.0), (22, 23, 1.0)], [(24, 25, 1.0)]]
    runs = [[30], [31]]
    infos = [(0, 100.0)]
    assert call_raw(board, runs, infos, 2, ph)[0] in (0, -5)               # valid (-5 without a GPU)
    assert call_raw(board, runs, infos, 2, ph, num_players=7)[0] == -1      # players out of range
    assert call_raw([0, 5, 10, 10], runs, infos, 2, ph)[0] == -1            # repeated board card
    assert call_raw(board, [[10]], infos, 2, ph)[0] == -1                   # runout card on the board
    assert call_raw(board, runs, infos, 2, [[(20, 20, 1.0)], [(24, 25, 1.0)]])[0] == -1   # hand with one card twice
    assert call_raw(board, runs, infos, 2, [[(20, 52, 1.0)], [(24, 25, 1.0)]])[0] == -1   # card outside the deck
    assert call_raw(board, runs, infos, 1, ph)[0] == -1                     # a range larger than max_hands
    rc, msg = call_raw(board, runs, [(-1, 100.0)], 2, ph)
    assert rc == -1 and "leaf_idx" in msg
    with pytest.raises(ValueError):
        lv.compute_turn_leaf_values(board, [], 2, 100)
    with pytest.raises(ValueError):
        lv.compute_flop_leaf_equity(board[:3], [], 2, 100, player_hands=[ph[0]])


@pytest.mark.skipif(HAVE_GPU, reason="checks the behaviour without a CUDA device")
def test_no_cpu_fallback_without_a_gpu():
    board = [0, 5, 10, 15]
    ph = [[(20, 21, 1.0), (22, 23, 1.0)], [(24, 25, 1.0)]]
    with pytest.raises(RuntimeError, match="ss_leaf_values_gpu failed"):
        lv.compute_turn_leaf_values(board, [lv.LeafInfo(0, 100, (10, 10))], 2, 100, player_hands=ph)


def test_descriptors_of_a_four_player_tree():
    cfg = wl.config("turn3", seed=24, num_hands=16, num_players=4, bet_sizes=[1.0], max_raises=1)
    cfg["hands"], cfg["weights"] = wl.make_ranges(np.random.default_rng(24), cfg["board"], 4, 16)
    sg = wl.AbiSubgame(cfg)
    try:
        got = lv.extract_leaf_info_from_tree(sg.td, 4)
        want = leaf_oracle.leaf_infos(sg.td, 4)
    finally:
        sg.free()
    assert len(got) > 0
    assert [(i.leaf_idx, i.pot, i.bets) for i in got] == want


@pytest.mark.parametrize("seed,num_board,players,hands", [
    (2, 4, 3, None),     # 3-player turn, 1128 hands: 12 river cards, 2000 sampled opponent pairs
    (5, 4, 6, 60),       # 6 players: 2000 sampled opponent 5-tuples
    (7, 3, 3, 30),       # 3-player flop, small ranges: every turn and river card
])
def test_element_functions_at_size_against_numpy_oracle(emul, tmp_path, seed, num_board, players, hands):
    rng = np.random.default_rng(seed)
    board = [int(c) for c in rng.permutation(52)[:num_board]]
    hs, ws = wl.make_ranges(rng, board, players, hands)
    ph = [[(int(h[0]), int(h[1]), float(w)) for h, w in zip(hs[p], ws[p])] for p in range(players)]
    infos = [(i, int(p)) for i, p in enumerate(rng.integers(60, 900, 3))]
    mh = max(len(h) for h in hs)
    runs = runouts_for(board, ph)
    want = leaf_oracle.leaf_values_vectorised(board, runs, [(i, p, ()) for i, p in infos], mh, ph)
    got = emulate(emul, tmp_path, board, runs, infos, mh, ph)
    assert np.array_equal(got, want)
