"""The reference data-flow bytes per iteration that bench.py reports beside
the kernel roofline (roofline_iteration), on the three benchmark trees:
heads-up river (51 nodes, 1081 hands), 3-player turn with continuation
leaves (21,436 nodes, 1128 hands), 6-player river (19,579 nodes, 1081
hands).  Trees come from the library's host-side builder; no GPU.  Also
the binding of the reference's CPU solver src/solver.c that the heads-up
river leg times as its baseline."""
import pytest

import workloads as wl


@pytest.fixture(scope="module")
def bench():
    import importlib
    import sys
    argv = sys.argv
    sys.argv = ["bench.py"]
    try:
        return importlib.import_module("bench")
    finally:
        sys.argv = argv


@pytest.mark.parametrize("name,over,H,nodes,want", [
    ("hu_river", {}, 1081, 51, 4_202_928),
    ("turn3", {}, 1128, 21_436, 3_152_399_040),
    ("river6", {}, 1081, 19_579, 8_289_419_328),
])
def test_flow_bytes(bench, name, over, H, nodes, want):
    cfg = wl.config(name, seed=0, **over)
    sg = wl.AbiSubgame(cfg, max_hands=1326)
    assert sg.td.num_nodes == nodes
    assert bench.flow_bytes_per_iteration(sg.td, H) == want
    sg.free()


def test_reference_cpu_solver_binding():
    """The heads-up river CPU baseline drives the reference's own src/solver.c
    (oracle/_ref/libref_solver.so) through its API: a small seeded solve."""
    from oracle.oracle import RefSolverC, ref_solver_available
    if not ref_solver_available():
        pytest.skip("reference solver build missing")
    import workloads as wl
    cfg = wl.config("hu_river", seed=3, num_hands=40)
    secs = RefSolverC().solve(cfg["board"], cfg["hands"], cfg["weights"], cfg["pot"], cfg["stack"],
                              cfg["bet_sizes"], 5)
    assert 0.0 < secs < 60.0
