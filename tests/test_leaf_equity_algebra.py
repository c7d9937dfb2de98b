"""The counting form a device leaf-value producer would use, checked on CPU
against the reference-generated fixtures (tests/golden/leaf_values_*.npz,
heads-up cases): per runout, a hand's wins and valid opponent hands are
  L = lt - lt_a - lt_b,   E = le - le_a - le_b + [opponent holds {a, b}] - L,
  V = n - n_a - n_b + [opponent holds {a, b}],
from the counts of the opponent's hands below (lt) / at or below (le) its
strength, overall and among those holding card a or b (sorted strengths
and a binary search, per card), instead of the reference's loop over every
opponent hand (python/leaf_values.py:573-691).  Wins L + E/2 and V are
sums of ones and halves, exact in FP64, so the values match bit for bit."""
import glob
import os
from collections import defaultdict

import numpy as np
import pytest

import workloads as wl
from oracle import leaf_oracle
from oracle.oracle import Oracle

HERE = os.path.dirname(os.path.abspath(__file__))
HU = [p for p in sorted(glob.glob(os.path.join(HERE, "golden", "leaf_values_*.npz")))
      if int(np.load(p)["num_players"]) == 2]


def counted_equity(board, runouts, hands, max_hands, orc):
    raw = np.zeros((2, max_hands))
    cnt = np.zeros((2, max_hands))
    for extra in runouts:
        b5 = list(board) + extra
        dead = set(b5)
        live = []
        for p in range(2):
            idx = [h for h, (c0, c1) in enumerate(hands[p]) if c0 not in dead and c1 not in dead]
            st = np.array([orc.eval7(b5 + [int(hands[p][h][0]), int(hands[p][h][1])]) for h in idx], np.int64)
            live.append((idx, st))
        for p in range(2):
            q = 1 - p
            qidx, qst = live[q]
            if not len(qidx):
                continue
            order = np.sort(qst)
            by_card = defaultdict(list)
            combos = set()
            for o, s in zip(qidx, qst):
                c0, c1 = int(hands[q][o][0]), int(hands[q][o][1])
                by_card[c0].append(s)
                by_card[c1].append(s)
                combos.add((min(c0, c1), max(c0, c1)))
            by_card = {c: np.sort(v) for c, v in by_card.items()}
            empty = np.zeros(0, np.int64)
            for h, s in zip(*live[p]):
                a, b = int(hands[p][h][0]), int(hands[p][h][1])
                ca, cb = by_card.get(a, empty), by_card.get(b, empty)
                both = 1 if (min(a, b), max(a, b)) in combos else 0
                lt = np.searchsorted(order, s, "left") - np.searchsorted(ca, s, "left") - np.searchsorted(cb, s, "left")
                le = (np.searchsorted(order, s, "right") - np.searchsorted(ca, s, "right")
                      - np.searchsorted(cb, s, "right") + both)
                n = len(order) - len(ca) - len(cb) + both
                if n > 0:
                    raw[p, h] += (lt + 0.5 * (le - lt)) / n
                    cnt[p, h] += 1.0
    ok = cnt > 0
    raw[ok] /= cnt[ok]
    return raw


@pytest.mark.parametrize("path", HU, ids=[os.path.basename(p)[12:-4] for p in HU])
def test_counting_form_matches_reference(path):
    g = np.load(path)
    board = [int(c) for c in g["board"]]
    hands = [g["hands"][p] for p in range(2)]
    ws = [g["weights"][p] for p in range(2)]
    mh = int(g["max_hands"])
    ph = [[(int(h[0]), int(h[1]), float(w)) for h, w in zip(hands[p], ws[p])] for p in range(2)]
    runouts = (leaf_oracle.turn_runouts if len(board) == 4 else leaf_oracle.flop_runouts)(board, ph)
    eq = counted_equity(board, runouts, hands, mh, Oracle())
    cfg = dict(board=board, pot=int(g["pot"]), stack=int(g["stack"]), bet_sizes=[float(x) for x in g["bet_sizes"]],
               max_raises=int(g["max_raises"]), num_players=2, hands=hands, weights=ws)
    sg = wl.AbiSubgame(cfg)
    infos = leaf_oracle.leaf_infos(sg.td, 2)
    sg.free()
    out = np.zeros_like(g["leaf_values"])
    for leaf, pot, _ in infos:
        for combo in range(16):
            prof = (combo % 4, combo // 4)
            for p in range(2):
                for h in range(len(hands[p])):
                    out[leaf * 16 + combo, p, h] = leaf_oracle.biased_value(eq[p, h], pot, prof[p], prof[1 - p])
    assert np.array_equal(out, g["leaf_values"])
