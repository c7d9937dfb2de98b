"""GPU continuation-value producer (ss_leaf_values_gpu) against the
reference and the oracle, through the host module
poker-solver_b200/leaf_values.py (the drop-in for python/leaf_values.py):
* the reference module's own outputs (tests/golden/leaf_values_*.npz:
  heads-up and 3-player turns, heads-up flops, every runout and sampled
  ones, enumerated and sampled opponent tuples), bit for bit;
* edge cases against the oracle's loop form: an empty range, a range the
  board blocks entirely, four players;
* full-size ranges (1128 combos on a turn, 3 and 4 players, a heads-up flop
  with 144 runouts, six players) against the oracle's numpy form, which is
  pinned to the same fixtures (tests/test_leaf_oracle.py), bit for bit;
* the leaf descriptors of the 3-player turn benchmark tree (21,436 nodes),
  whose values fill 126 MB, against the same oracle, twice in a row.
Collected after the solver's GPU tests (tests/conftest.py)."""
import numpy as np
import pytest

import leaf_values as lv
import workloads as wl
from oracle import leaf_oracle
from test_leaf_producer import FIXTURES, IDS, edge_cases, load_case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("path", FIXTURES, ids=IDS)
def test_reference_fixtures_bit_for_bit(path):
    g, board, _, _, ph, infos = load_case(path)
    infos = [lv.LeafInfo(i, p, ()) for i, p in infos]
    produce = lv.compute_turn_leaf_values if len(board) == 4 else lv.compute_flop_leaf_equity
    got = produce(board, infos, int(g["max_hands"]), int(g["pot"]), player_hands=ph)
    assert got.dtype == np.float32 and got.shape == g["leaf_values"].shape
    assert np.array_equal(got, g["leaf_values"])


def test_legacy_two_player_arguments():
    g, board, _, _, ph, infos = load_case([p for p in FIXTURES if "hu_small" in p and "flop" not in p][0])
    infos = [lv.LeafInfo(i, p, ()) for i, p in infos]
    got = lv.compute_turn_leaf_values(board, infos, int(g["max_hands"]), int(g["pot"]), oop_hands=ph[0], ip_hands=ph[1])
    assert np.array_equal(got, g["leaf_values"])


@pytest.mark.parametrize("case", edge_cases(), ids=lambda c: c[0])
def test_edge_cases_against_oracle(case):
    _, board, ph, infos, mh = case
    got = lv.compute_turn_leaf_values(board, [lv.LeafInfo(i, p, ()) for i, p in infos], mh, 100, player_hands=ph)
    want = leaf_oracle.turn_leaf_values(board, [(i, p, ()) for i, p in infos], mh, ph)
    assert np.array_equal(got, want)


def full_case(seed, num_board, players, hands):
    rng = np.random.default_rng(seed)
    board = [int(c) for c in rng.permutation(52)[:num_board]]
    hs, ws = wl.make_ranges(rng, board, players, hands)
    ph = [[(int(h[0]), int(h[1]), float(w)) for h, w in zip(hs[p], ws[p])] for p in range(players)]
    infos = [(i, int(p)) for i, p in enumerate(rng.integers(60, 900, 7))]
    return board, ph, infos, max(len(h) for h in hs)


@pytest.mark.parametrize("name,seed,num_board,players,hands", [
    ("hu_turn_1128", 1, 4, 2, None),
    ("three_turn_1128", 2, 4, 3, None),
    ("hu_flop_400", 3, 3, 2, 400),
    ("four_turn_300", 4, 4, 4, 300),
    ("six_turn_60", 5, 4, 6, 60),
])
def test_full_size_against_oracle(name, seed, num_board, players, hands):
    board, ph, infos, mh = full_case(seed, num_board, players, hands)
    runouts = (lv.turn_runouts if num_board == 4 else lv.flop_runouts)(board, [len(h) for h in ph])
    want = leaf_oracle.leaf_values_vectorised(board, runouts, [(i, p, ()) for i, p in infos], mh, ph)
    produce = lv.compute_turn_leaf_values if num_board == 4 else lv.compute_flop_leaf_equity
    got = produce(board, [lv.LeafInfo(i, p, ()) for i, p in infos], mh, 100, player_hands=ph)
    assert np.array_equal(got, want)


def test_turn_benchmark_tree_twice():
    cfg = wl.config("turn3", seed=0)
    sg = wl.AbiSubgame(cfg)
    try:
        infos = lv.extract_leaf_info_from_tree(sg.td, cfg["num_players"])
    finally:
        sg.free()
    ph = [[(int(h[0]), int(h[1]), float(w)) for h, w in zip(cfg["hands"][p], cfg["weights"][p])]
          for p in range(cfg["num_players"])]
    mh = max(len(h) for h in ph)
    first = lv.compute_turn_leaf_values(cfg["board"], infos, mh, cfg["pot"], player_hands=ph)
    second = lv.compute_turn_leaf_values(cfg["board"], infos, mh, cfg["pot"], player_hands=ph)
    runouts = lv.turn_runouts(cfg["board"], [len(h) for h in ph])
    want = leaf_oracle.leaf_values_vectorised(cfg["board"], runouts, [(i.leaf_idx, i.pot, ()) for i in infos], mh, ph)
    assert first.shape == (len(infos) * 64, 3, mh)
    assert np.array_equal(first, want)
    assert np.array_equal(second, first)
