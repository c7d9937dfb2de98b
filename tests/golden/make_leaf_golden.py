"""Generate the leaf-value golden fixtures (tests/golden/leaf_values_*.npz)
from the reference's own producers, python/leaf_values.py
(compute_turn_leaf_values, compute_flop_leaf_equity and
extract_leaf_info_from_tree), imported from the reference sources, on
seeded turn and flop subgames whose trees come from this library's
ss_build_tree.  Each fixture stores the subgame (board, pot,
stack, bet sizes, raise cap, ranges), the reference's leaf descriptors and
its leaf values.  The script also checks that the reference module's own
7-card evaluator orders hands as the oracle's evaluator (pinned to
src/hand_eval.h) does, on random showdowns.

Usage (needs the reference sources, i.e. this container):
    python tests/golden/make_leaf_golden.py [reference root]
"""
import importlib.util
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "poker-solver_b200")]

import workloads as wl  # noqa: E402
from oracle.oracle import Oracle  # noqa: E402

def _ref_root():
    """The reference checkout: argv[1], else the one place it is configured
    (oracle/build_ref.py: REF_ROOT or its default location)."""
    if len(sys.argv) > 1:
        return sys.argv[1]
    spec = importlib.util.spec_from_file_location("oracle_build_ref", os.path.join(ROOT, "oracle", "build_ref.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.REF


REF = _ref_root()

# name, seed, board cards, players, hands per player, bet sizes, raise cap
CASES = [
    ("hu_small", 201, 4, 2, 30, [1.0], 1),        # every river card, every opponent hand
    ("hu_sampled", 202, 4, 2, 60, [0.75], 1),     # 12 sampled river cards
    ("three_small", 203, 4, 3, 10, [1.0], 1),     # opponent pairs enumerated
    ("three_sampled", 204, 4, 3, 52, [1.0], 1),   # 2000 sampled opponent pairs, 12 rivers
    ("flop_hu_small", 205, 3, 2, 16, [1.0], 1),   # every turn and river card
    ("flop_hu_sampled", 206, 3, 2, 56, [1.0], 1), # 12 x 12 sampled runouts
]


def load_reference():
    spec = importlib.util.spec_from_file_location("ref_leaf_values", os.path.join(REF, "python", "leaf_values.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def check_evaluators(ref, orc, rng, n=4000):
    deck = np.arange(52)
    for _ in range(n):
        c = rng.permutation(deck)[:9].tolist()
        board, h1, h2 = c[:5], c[5:7], c[7:9]
        r1, r2 = ref._eval7_py(board + h1), ref._eval7_py(board + h2)
        o1, o2 = orc.eval7(board + h1), orc.eval7(board + h2)
        if (r1 > r2) != (o1 > o2) or (r1 == r2) != (o1 == o2):
            raise AssertionError(f"evaluators disagree on {board} {h1} {h2}")


def main():
    ref = load_reference()
    orc = Oracle()
    check_evaluators(ref, orc, np.random.default_rng(7))
    for name, seed, nb, np_, nh, sizes, raises in CASES:
        rng = np.random.default_rng(seed)
        board = [int(x) for x in rng.permutation(52)[:nb]]
        hands, ws = wl.make_ranges(rng, board, np_, nh)
        cfg = dict(board=board, pot=120, stack=480, bet_sizes=sizes, max_raises=raises, num_players=np_,
                   hands=hands, weights=ws)
        sg = wl.AbiSubgame(cfg)
        infos = ref.extract_leaf_info_from_tree(sg.td, np_)
        ph = [[(int(h[0]), int(h[1]), float(w)) for h, w in zip(hands[p], ws[p])] for p in range(np_)]
        mh = max(len(h) for h in hands)
        produce = ref.compute_turn_leaf_values if nb == 4 else ref.compute_flop_leaf_equity
        lv = produce(board, infos, mh, 120, player_hands=ph)
        np.savez_compressed(
            os.path.join(HERE, f"leaf_values_{name}.npz"),
            board=np.array(board, np.int32), pot=120, stack=480, bet_sizes=np.array(sizes, np.float32),
            max_raises=raises, num_players=np_, max_hands=mh,
            hands=np.stack([np.asarray(h, np.int32) for h in hands]),
            weights=np.stack([np.asarray(w, np.float32) for w in ws]),
            leaf_idx=np.array([li.leaf_idx for li in infos], np.int32),
            leaf_pot=np.array([li.pot for li in infos], np.int32),
            leaf_bets=np.array([li.bets for li in infos], np.int32),
            leaf_values=np.asarray(lv, np.float32))
        sg.free()
        print(f"{name}: {len(infos)} leaves, values {lv.shape}")


if __name__ == "__main__":
    main()
