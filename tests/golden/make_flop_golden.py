"""Golden vectors of the reference's multi-street solve, made by its own
sm_100a build of src/cuda/flop_solve.cu (oracle/_ref/libref_flop_solve_gpu.so,
oracle/build_ref.py) on a B200:

    python tests/golden/make_flop_golden.py [OUTDIR]      # default tests/golden

For each seeded case: the inputs (flop, pot, stack, bet sizes, hands,
weights) and the root strategy of fs_solve_gpu after 1, 2, 3 and 5
iterations.  (The reference's fs_solve_gpu_extract_all cannot be used: it
allocates room for 52 turn roots, flop_solve.cu:1529-1530, and writes one
per card under every flop-ending chance node -- 245 on these trees --
corrupting the host heap.)
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
    # name, seed, flop, pot, stack, bet sizes, hands per player
    ("small", 301, [0, 13, 26], 1000, 5000, [0.75], 10),
    ("two_sizes", 302, [51, 7, 22], 650, 9750, [0.5, 1.0], 14),
    ("wide", 303, [4, 30, 45], 400, 2000, [1.0], 60),
]
ITERATIONS = (1, 2, 3, 5)


def main():
    out_dir = sys.argv[1] if len(sys.argv) > 1 else HERE
    os.makedirs(out_dir, exist_ok=True)
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_flop_solve_gpu.so"))
    for name, seed, flop, pot, stack, sizes, nh in CASES:
        h, w = wl.make_ranges(np.random.default_rng(seed), flop, 2, nh)
        sg = fsm.FlopSubgame(lib, flop, pot, stack, sizes, h, w)
        n = sg.td.num_nodes
        roots = {f"root_strategy_{k}": sg.solve(k)["root_strategy"] for k in ITERATIONS}
        sg.free()
        np.savez_compressed(os.path.join(out_dir, f"flop_ref_{name}.npz"), flop=np.array(flop), pot=pot,
                            stack=stack, bet_sizes=np.array(sizes, np.float32), hands=np.array(h, np.int32),
                            weights=np.array(w, np.float32), iterations=np.array(ITERATIONS), num_nodes=n, **roots)
        print(name, "nodes", n)


if __name__ == "__main__":
    main()
