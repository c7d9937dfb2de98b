"""Generate the golden fixtures of tests/golden/ from the reference itself.

Runs the reference solver src/cuda/street_solve.cu (its own kernels, compiled
for the host by oracle/build_ref.py into oracle/_ref/) and the reference hand
evaluator src/hand_eval.h on small seeded cases, and stores inputs and outputs:

  ref_solve_*.npz      tree arrays, ranges, leaf values, frozen actions and the
                       reference outputs (root strategy, root values, average
                       strategies) after a fixed number of iterations
  hand_rank_all.json   checksum over all C(52,7) 7-card sets of
                       mix64(card mask) * strength (mod 2^64) and the
                       per-category counts
  hand_rank_sample.npz 20,000 random 7-card hands with their strengths

Usage (needs the reference sources, i.e. this container):
    python oracle/build_ref.py && python tests/golden/make_golden.py
"""
import ctypes
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "poker-solver_b200")]

from oracle.oracle import RefHandEval, RefStreetSolve  # noqa: E402
import workloads as wl  # noqa: E402

# name, workload, seed, hands/player, players, board cards, iterations, raise cap,
# bet sizes, freeze root action
CASES = [
    ("hu_river", "hu_river", 101, 20, 2, 5, 30, 2, [0.5, 1.0], None),
    ("hu_turn", "hu_river", 102, 16, 2, 4, 10, 3, [0.5, 1.0], None),
    ("river3", "river6", 103, 8, 3, 5, 4, 2, [0.5, 1.0], None),
    ("turn3", "turn3", 104, 8, 3, 4, 4, 3, [0.75], None),
    ("hu_river_frozen", "hu_river", 105, 20, 2, 5, 12, 2, [0.5, 1.0], 1),
]


def main():
    for name, wname, seed, nh, np_, nb, iters, raises, sizes, freeze in CASES:
        cfg = wl.config(wname, seed=seed, num_hands=nh, num_players=np_, max_raises=raises,
                        bet_sizes=sizes)
        cfg["board"] = cfg["board"][:nb]
        cfg["hands"], cfg["weights"] = wl.make_ranges(np.random.default_rng(seed), cfg["board"], np_, nh)
        ref = RefStreetSolve(200, raises, "cpu")
        td = ref.build(cfg["board"], cfg["pot"], cfg["stack"], sizes, np_)
        tree = ref.tree(td)
        lv = wl.leaf_values_for(cfg, td.num_leaves)
        frozen = None
        if freeze is not None:
            frozen = np.full(tree.num_nodes, -1, np.int32)
            frozen[0] = freeze
        H, W, n = wl.padded(cfg)
        out = ref.solve(td, H, W, n, iters, leaf_values=lv, frozen=frozen)
        ref.free(td)
        np.savez_compressed(
            os.path.join(HERE, f"ref_solve_{name}.npz"),
            board=np.array(cfg["board"], np.int32), pot=cfg["pot"], stack=cfg["stack"],
            bet_sizes=np.array(sizes, np.float32), max_raises=raises, num_players=np_,
            iterations=iters, hands=H, weights=W, num_hands=n,
            leaf_values=lv if lv is not None else np.zeros(0, np.float32),
            frozen=frozen if frozen is not None else np.zeros(0, np.int32),
            nodes=tree.nodes, children=tree.children, level_order=tree.level_order,
            node_depth=tree.node_depth, max_depth=tree.max_depth, num_leaves=tree.num_leaves,
            **{k: out[k] for k in ("root_strategy", "root_ev", "avg_strategies", "avg_node_ids")},
            root_player=out["root_player"], root_num_actions=out["root_num_actions"])
        print("wrote", name, tree.num_nodes, "nodes")

    he = RefHandEval()
    he.lib.ref_eval7_checksum.restype = ctypes.c_uint64
    hist = (ctypes.c_uint64 * 10)()
    chk = he.lib.ref_eval7_checksum(hist)
    json.dump({"checksum": f"{chk:#018x}", "category_counts": list(hist), "sets": int(sum(hist))},
              open(os.path.join(HERE, "hand_rank_all.json"), "w"), indent=1)
    rng = np.random.default_rng(7)
    cards = np.array([rng.choice(52, 7, replace=False) for _ in range(20000)], np.int32)
    np.savez_compressed(os.path.join(HERE, "hand_rank_sample.npz"), cards=cards,
                        strength=he.eval7_many(cards))
    print("wrote hand rank fixtures", f"{chk:#018x}")


if __name__ == "__main__":
    main()
