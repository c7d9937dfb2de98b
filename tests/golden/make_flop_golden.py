"""Golden vectors of the reference's multi-street solve, made by its own
sm_100a build of src/cuda/flop_solve.cu (oracle/_ref/libref_flop_solve_gpu.so,
oracle/build_ref.py) on a B200:

    python tests/golden/make_flop_golden.py [OUTDIR]      # default tests/golden

For each seeded case: the inputs (flop, pot, stack, bet sizes, hands,
weights, iterations), the root strategy of fs_solve_gpu, and the normalised
average strategies and values of fs_solve_gpu_extract_all at a sample of
node ids (the first 400, every 1009th, and the turn roots; the whole tree
holds ~575 K nodes).
"""
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "poker-solver_b200")]

import flop_solve as fsm  # noqa: E402
import workloads as wl  # noqa: E402

CASES = [
    # name, seed, flop, pot, stack, bet sizes, hands per player, iterations
    ("small", 301, [0, 13, 26], 1000, 5000, [0.75], 10, 4),
    ("two_sizes", 302, [51, 7, 22], 650, 9750, [0.5, 1.0], 14, 3),
    ("wide", 303, [4, 30, 45], 400, 2000, [1.0], 60, 2),
]


def sample_nodes(n, roots):
    ids = set(range(min(400, n))) | set(range(0, n, 1009)) | set(int(r) for r in roots)
    return np.array(sorted(ids), np.int32)


def main():
    out_dir = sys.argv[1] if len(sys.argv) > 1 else HERE
    os.makedirs(out_dir, exist_ok=True)
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_flop_solve_gpu.so"))
    for name, seed, flop, pot, stack, sizes, nh, iters in CASES:
        h, w = wl.make_ranges(np.random.default_rng(seed), flop, 2, nh)
        sg = fsm.FlopSubgame(lib, flop, pot, stack, sizes, h, w)
        n = sg.td.num_nodes
        r = sg.solve(iters, extract=True)
        ids = sample_nodes(n, r["turn_root_indices"])
        np.savez_compressed(os.path.join(out_dir, f"flop_ref_{name}.npz"), flop=np.array(flop), pot=pot,
                            stack=stack, bet_sizes=np.array(sizes, np.float32), hands=np.array(h, np.int32),
                            weights=np.array(w, np.float32), iterations=iters, root_strategy=r["root_strategy"],
                            node_ids=ids, avg=r["all_avg_strategies"][ids], cfv=r["all_cfv"][ids],
                            turn_root_indices=r["turn_root_indices"], turn_root_cards=r["turn_root_cards"],
                            num_nodes=n)
        sg.free()
        print(name, "nodes", n, "sampled", len(ids))


if __name__ == "__main__":
    main()
