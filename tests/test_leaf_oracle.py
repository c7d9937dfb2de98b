"""The oracle's restatement of the reference's turn and flop leaf-value
producers (oracle/leaf_oracle.py) against golden vectors made by the
reference module itself (tests/golden/make_leaf_golden.py): leaf descriptors
read from this library's trees and the leaf values, bit for bit, on
heads-up and 3-player turns and heads-up flops, with every runout and every
opponent tuple, and with the reference's sampled runouts and sampled
opponent pairs."""
import glob
import os

import numpy as np
import pytest

import workloads as wl
from oracle import leaf_oracle

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "leaf_values_*.npz")))


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p)[12:-4] for p in FIXTURES])
def test_leaf_values_match_reference(path):
    g = np.load(path)
    np_ = int(g["num_players"])
    board = [int(c) for c in g["board"]]
    hands = [g["hands"][p] for p in range(np_)]
    ws = [g["weights"][p] for p in range(np_)]
    cfg = dict(board=board, pot=int(g["pot"]), stack=int(g["stack"]), bet_sizes=[float(x) for x in g["bet_sizes"]],
               max_raises=int(g["max_raises"]), num_players=np_, hands=hands, weights=ws)
    sg = wl.AbiSubgame(cfg)
    infos = leaf_oracle.leaf_infos(sg.td, np_)
    sg.free()
    assert [i[0] for i in infos] == g["leaf_idx"].tolist()
    assert [i[1] for i in infos] == g["leaf_pot"].tolist()
    assert [list(i[2]) for i in infos] == g["leaf_bets"].tolist()
    ph = [[(int(h[0]), int(h[1]), float(w)) for h, w in zip(hands[p], ws[p])] for p in range(np_)]
    produce = leaf_oracle.turn_leaf_values if len(board) == 4 else leaf_oracle.flop_leaf_values
    got = produce(board, infos, int(g["max_hands"]), ph)
    assert got.shape == g["leaf_values"].shape
    assert np.array_equal(got, g["leaf_values"])


def test_fixtures_present():
    assert len(FIXTURES) >= 6


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p)[12:-4] for p in FIXTURES])
def test_vectorised_form_matches_reference(path):
    """The numpy form of the oracle (used at full size by the GPU tests)
    against the same reference-generated fixtures, bit for bit."""
    g = np.load(path)
    np_ = int(g["num_players"])
    board = [int(c) for c in g["board"]]
    ph = [[(int(h[0]), int(h[1]), float(w)) for h, w in zip(g["hands"][p], g["weights"][p])] for p in range(np_)]
    infos = [(int(i), int(pot), ()) for i, pot in zip(g["leaf_idx"], g["leaf_pot"])]
    runouts = (leaf_oracle.turn_runouts if len(board) == 4 else leaf_oracle.flop_runouts)(board, ph)
    got = leaf_oracle.leaf_values_vectorised(board, runouts, infos, int(g["max_hands"]), ph)
    assert np.array_equal(got, g["leaf_values"])
