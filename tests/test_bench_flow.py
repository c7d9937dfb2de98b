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


def test_ncu_summary_classes(bench, tmp_path):
    """bench.py --ncu-summary: launches are matched to profile classes by their
    base function name, whether ncu prints the demangled signature or the bare
    name; each class keeps its mean DRAM bytes (read + write) per launch, and
    the file is stamped with the kernel sources' hash."""
    import csv
    import json
    head = ["ID", "Process ID", "Process Name", "Host Name", "Kernel Name", "Context", "Stream", "Block Size",
            "Grid Size", "Device", "CC", "Section Name", "Metric Name", "Metric Unit", "Metric Value"]
    launches = [
        ("0", "void unnamed>::k_term_cr2<float>(DevCtx, const DevCtx *, const TermItem *, const int *, int)",
         1000, 300),
        ("1", "void unnamed>::k_term_cr2<float>(DevCtx, const DevCtx *, const TermItem *, const int *, int)",
         3000, 700),
        ("2", "void ssb::(anonymous namespace)::k_cfv<1>(DevCtx, const DevCtx *, const CfvItem *, int, int, int)",
         500, 0),
        ("3", "k_reach", "1,024", 0),
        ("4", "cutlass_kernel_not_ours", 9, 9),
    ]
    rows = [head]
    for i, name, rd, wr in launches:
        for metric, v in (("dram__bytes_read.sum", rd), ("dram__bytes_write.sum", wr),
                          ("gpu__time_duration.sum", 10)):
            rows.append([i, "1", "python3", "127.0.0.1", name, "1", "7", "(256, 1, 1)", "(8, 1, 1)", "0", "10.0",
                         "Command line profiler metrics", metric, "byte", str(v)])
    src = tmp_path / "launches.csv"
    with open(src, "w", newline="") as f:
        f.write("==PROF== Connected to process 1\n")
        csv.writer(f).writerows(rows)
    out = tmp_path / "dram_traffic.json"
    bench.ncu_summary(str(src), "turn3", "ncu ...", path=str(out))
    tr = json.load(open(out))
    assert tr["kernel_sources_sha16"] == bench.kernel_sources_sha16()
    cls = tr["workloads"]["turn3"]["classes"]
    assert cls == {"term_cr2": {"launches_captured": 2, "dram_bytes_per_launch": 2500},
                   "cfv": {"launches_captured": 1, "dram_bytes_per_launch": 500},
                   "reach": {"launches_captured": 1, "dram_bytes_per_launch": 1024}}
