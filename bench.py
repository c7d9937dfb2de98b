"""Benchmark: subgame solves/s (and p50/p99 latency) of the B200 street solver.

Workload (one step = one full solve): the 3-player turn subgame with
depth-limited leaves -- seeded 4-card board, all 1128 non-board combos per
player with weights U(0,1) and ~30% zeroed, pot 150, stacks 500, bets
{0.33, 0.75, 1.5 pot, all-in}, 3 raises, continuation leaves with per-hand
values N(0, 0.3 pot); 1000 Linear-CFR iterations in FP32 (21,436 nodes,
15,616 leaves).  Synthetic seeded inputs stand in for the reference's
realtime requests; there is no dataset.

  value  -- solves/s with the subgame resident in HBM (ss_session_reset +
            ss_session_run), timed with CUDA events on the session's stream
  e2e    -- solves/s through the reference-facing C ABI (ss_solve_gpu) from a
            host-built tree: tables, ranges and leaf values host->device,
            average strategies device->host, inside the timed region
N GPUs (torchrun): every rank solves its own seeded subgames (weak scaling,
no data-path collective); the step time is the max over ranks.

--impl reference times the reference's own implementation of this path on
the host cores: src/cuda/street_solve.cu with its kernels run on the CPU
(oracle/_ref, built by oracle/build_ref.py).  Its tuple enumeration is
O(H^3) per leaf and hand for three players, so each step is a bounded sample
(one iteration of the full tree at small range sizes, all cores busy) whose
full-size rate is extrapolated with the fitted size exponent; the line
reports the median over the steps.
"""
import argparse
import ctypes
import json
import os
import re
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "poker-solver_b200")
sys.path[:0] = [ROOT, PKG]

METRIC = "subgame solves/s and p50/p99 latency at <=0.5% pot exploitability vs plain GPU"
UNIT = "solves/s"
WORKLOAD = "turn3"
# --workload: the benchmark's subgame (turn3 by default) or the 3-player river
WORKLOADS = {
    "turn3": ("3-player turn subgame, 1128 combos/player, continuation leaves, 1000 Linear-CFR iterations",
              "state larger than L2 (regrets, sums, reach, values ~400 MB)"),
    "river3": ("3-player river subgame, 1081 combos/player with U(0,1) weights, pot 300, stacks 1000, "
               "bets {0.5, 1.0} + all-in, 2 raises, three-way showdowns, 1000 Linear-CFR iterations",
               "state a few MB, inside L2"),
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--iterations", type=int, default=1000)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--workload", default=WORKLOAD, choices=sorted(WORKLOADS),
                    help="subgame of the plain form (the CPU baseline and reference arm cover turn3)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--forms", default="plain,batched,served,hu_river,leaf,four,anchor,flop",
                    help="comma list of plain (the headline), batched, served, hu_river (the heads-up river "
                         "beside the reference's CPU solver), leaf (the turn subgame's continuation values "
                         "produced on the GPU), four (full-range 4-player turn and river, three-opponent "
                         "terminals)")
    ap.add_argument("--batch-size", type=int, default=512, help="batched form: mixed requests in one batch")
    ap.add_argument("--rates", default="50,500,2000", help="served form: request rates per second")
    ap.add_argument("--served-requests", type=int, default=256, help="served form: requests per rate")
    ap.add_argument("--ncu-summary", nargs=2, metavar=("CSV", "COMMAND"),
                    help="no run: summarise an ncu launch list (DRAM bytes per launch and class) of the "
                         "--workload into profiles/dram_traffic.json, stamped with the kernel sources' hash")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# distributed plumbing
# ---------------------------------------------------------------------------

def dist_init():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        backend = "nccl" if _cuda_ok() else "gloo"
        if backend == "nccl":
            import torch
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def _cuda_ok():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def dist_max(x):
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return x
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_sum(x):
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return x
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.barrier()


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------

class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx = max(mx, float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# our solver
# ---------------------------------------------------------------------------

def build_subgame(seed, iterations, workload=WORKLOAD):
    import workloads as wl
    if workload == "river3":
        cfg = wl.config("river6", seed=seed, num_players=3, iterations=iterations)
        cfg["hands"], cfg["weights"] = wl.make_ranges(np.random.default_rng(seed), cfg["board"], 3, None)
    else:
        cfg = wl.config(WORKLOAD, seed=seed, iterations=iterations)
    sg = wl.AbiSubgame(cfg, max_hands=1326)
    sg.set_leaf_values(wl.leaf_values_for(cfg, sg.num_leaves))
    return cfg, sg


def flow_bytes_per_iteration(td, H):
    """FP32 bytes one CFR iteration of the reference's data flow moves on this
    tree with H hands per player (street_solve.cu:1471-1550), summed over the
    traversers t; for each decision node with A actions: regret matching
    (regrets read, strategy written) 8 A H; reach of every player rp != t
    (parent row read, A child rows written, plus the strategy read at rp's
    own nodes) 4 H + 4 A H (+ 4 A H); values (A child rows read, one row
    written, plus strategy read and regret / strategy-sum read-modify-write
    at t's nodes) 4 A H + 4 H (+ 20 A H); each terminal: the counted
    opponents' reach rows and the value row 4 H (k + 1), plus k + 1 rank rows
    at showdowns and the leaf-value row at leaves."""
    np_ = td.num_players_field
    typ, ply, nch, act = [], [], [], []
    for i in range(td.num_nodes):
        n = td.nodes[i]
        typ.append(n.type)
        ply.append(n.player)
        nch.append(n.num_children)
        act.append([n.active_players[o] for o in range(np_)])
    total = 0
    for t in range(np_):
        for ty, p, A, ac in zip(typ, ply, nch, act):
            if ty == 0:
                total += 8 * A * H
                total += (np_ - 1) * (4 * H + 4 * A * H) + (4 * A * H if p != t else 0)
                total += 4 * A * H + 4 * H + (20 * A * H if p == t else 0)
            else:
                k = np_ - 1 if ty == 1 else sum(1 for o in range(np_) if o != t and ac[o])
                total += 4 * H * (k + 1)
                if ty == 2:
                    total += 4 * H * (k + 1)
                elif ty == 4:
                    total += 4 * H
    return total


KERNEL_SOURCES = ("ss_kernels.cu", "ss_cr3.cuh", "ss_cr2_tc.cuh", "ss_rank.cuh", "ss_kernels.h", "ss_engine.h",
                  "ss_plan.cpp")
# kernel name prefix -> profile class of ss_session_profile
NCU_CLASSES = [("k_term_cr2", "term_cr2"), ("k_term_cr1", "term_cr1"), ("k_term_sd", "term_sd"),
               ("k_term_enum", "term_enum"), ("k_term_cr3", "term_enum"), ("k_term_fill", "term_fill"),
               ("k_cfv", "cfv"), ("k_reach", "reach")]


def kernel_sources_sha16():
    """Hash of the kernel sources, stamped on the DRAM-traffic capture so that
    a capture of older kernels is not reported as this build's traffic."""
    import hashlib
    h = hashlib.sha256()
    for name in KERNEL_SOURCES:
        with open(os.path.join(PKG, "csrc", name), "rb") as f:
            h.update(f.read())
    return h.hexdigest()[:16]


def ncu_summary(csv_path, workload, command, path=None):
    """Per profile class: launches captured and mean DRAM bytes (read + write)
    per launch, from an ncu --csv launch list with dram__bytes_read.sum and
    dram__bytes_write.sum; merged into path (profiles/dram_traffic.json)."""
    import csv
    per = {}
    with open(csv_path) as f:
        rows = [r for r in csv.reader(f) if len(r) > 5]
    head = rows[0]
    ki, mi, vi, ii = head.index("Kernel Name"), head.index("Metric Name"), head.index("Metric Value"), head.index("ID")
    launch = {}
    for r in rows[1:]:
        if r[mi] not in ("dram__bytes_read.sum", "dram__bytes_write.sum", "gpu__time_duration.sum"):
            continue
        d = launch.setdefault(r[ii], {"name": r[ki]})
        d[r[mi]] = float(r[vi].replace(",", ""))
    for d in launch.values():
        # ncu prints the demangled signature ("void ...::k_term_cr2<float>(...)")
        # or, with --print-kernel-base function, the bare name
        m = re.search(r"(?:^|[\s:])(k_\w+)", d["name"])
        base = m.group(1) if m else d["name"]
        cls = next((c for p, c in NCU_CLASSES if base.startswith(p)), None)
        if cls is None:
            continue
        e = per.setdefault(cls, {"launches_captured": 0, "bytes": 0.0})
        e["launches_captured"] += 1
        e["bytes"] += d.get("dram__bytes_read.sum", 0.0) + d.get("dram__bytes_write.sum", 0.0)
    path = path or os.path.join(ROOT, "profiles", "dram_traffic.json")
    try:
        tr = json.load(open(path))
    except Exception:
        tr = {}
    if tr.get("kernel_sources_sha16") != kernel_sources_sha16():
        tr = {"workloads": {}}
    tr["kernel_sources_sha16"] = kernel_sources_sha16()
    tr["source"] = command
    tr.setdefault("workloads", {})[workload] = {"classes": {
        c: {"launches_captured": e["launches_captured"],
            "dram_bytes_per_launch": int(round(e["bytes"] / e["launches_captured"]))}
        for c, e in sorted(per.items())}}
    with open(path, "w") as f:
        json.dump(tr, f, indent=1)
    return tr


def run_ours(args, world, rank, local):
    import torch
    import street_solver_gpu as ssg

    torch.cuda.set_device(local)
    lib = ssg.load_library(1326)
    lib.ss_session_create.restype = ctypes.c_int
    lib.ss_session_run.restype = ctypes.c_int
    lib.ss_session_reset.restype = ctypes.c_int
    lib.ss_session_synchronize.restype = ctypes.c_int
    lib.ss_session_profile.restype = ctypes.c_int
    lib.ss_session_stream.restype = ctypes.c_void_p
    lib.ss_session_stream.argtypes = [ctypes.c_void_p]
    lib.ss_session_destroy.argtypes = [ctypes.c_void_p]
    for f in ("ss_session_run", "ss_session_reset", "ss_session_synchronize"):
        getattr(lib, f).argtypes = [ctypes.c_void_p] + ([ctypes.c_int] if f == "ss_session_run" else [])

    cfg, sg = build_subgame(args.seed + rank, args.iterations, args.workload)
    opts = ssg.SSSolveOptions(local, 10, -1.0, 50, 0)
    sess = ctypes.c_void_p()
    rc = lib.ss_session_create(ctypes.byref(sg.td), ctypes.byref(opts), ctypes.byref(sess))
    if rc != 0:
        raise RuntimeError(f"ss_session_create failed ({rc}): {ssg.last_error(lib)}")

    class Prof(ctypes.Structure):
        _fields_ = [("num_classes", ctypes.c_int), ("name", (ctypes.c_char * 16) * 8),
                    ("launches", ctypes.c_int * 8), ("ms", ctypes.c_double * 8),
                    ("bytes", ctypes.c_double * 8), ("iteration_ms", ctypes.c_double)]

    def check(rc, what):
        if rc != 0:
            raise RuntimeError(f"{what} failed ({rc}): {ssg.last_error(lib)}")

    class LaunchRec(ctypes.Structure):
        _fields_ = [("cls", ctypes.c_int), ("items", ctypes.c_int), ("ms", ctypes.c_double),
                    ("bytes", ctypes.c_double)]

    # one profiled iteration (graph with event nodes between kernel classes),
    # half-way through a solve, where reach rows and regrets look like the
    # average timed iteration's (the first iteration's uniform strategies
    # leave no zero reach)
    check(lib.ss_session_reset(sess), "reset")
    check(lib.ss_session_run(sess, max(1, args.iterations // 2)), "run")
    prof = Prof()
    check(lib.ss_session_profile(sess, ctypes.byref(prof)), "profile")
    classes, cls_names = {}, []
    for k in range(prof.num_classes):
        name = bytes(prof.name[k]).split(b"\0")[0].decode()
        cls_names.append(name)
        classes[name] = {"launches": prof.launches[k], "ms": prof.ms[k], "bytes": prof.bytes[k]}
    nrec = ctypes.c_int(0)
    recs = (LaunchRec * 4096)()
    lib.ss_session_profile_launches.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                                ctypes.POINTER(ctypes.c_int)]
    check(lib.ss_session_profile_launches(sess, recs, 4096, ctypes.byref(nrec)), "profile launches")
    # per launch in launch order: class, work items, device us, GB/s of the bytes it must move
    launch_list = [[cls_names[r.cls], r.items, round(r.ms * 1e3, 1),
                    round(r.bytes / (r.ms / 1e3) / 1e9, 1) if r.ms > 0 else 0.0]
                   for r in recs[:min(nrec.value, 4096)] if r.items > 0]
    launches_per_iter = sum(v["launches"] for v in classes.values())
    reach_launches = classes["reach"]["launches"]

    stream = torch.cuda.ExternalStream(lib.ss_session_stream(sess), device=local)

    def step():
        check(lib.ss_session_reset(sess), "reset")
        check(lib.ss_session_run(sess, args.iterations), "run")

    for _ in range(args.warmup):
        step()
    check(lib.ss_session_synchronize(sess), "sync")

    clocks = ClockSampler(local)
    clocks.start()
    times = []
    barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev_end = torch.cuda.Event(enable_timing=True)
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    ev0.record(stream)
    evs[0].record(stream)
    for i in range(args.steps):
        step()
        evs[i + 1].record(stream)
    ev_end.record(stream)
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    # FP64 exploitability of the last solve's average strategy
    lib.ss_session_exploitability.restype = ctypes.c_int
    lib.ss_session_exploitability.argtypes = [ctypes.c_void_p] + [ctypes.POINTER(ctypes.c_double)] * 5
    expl, nash = ctypes.c_double(-1), ctypes.c_double(-1)
    erc = lib.ss_session_exploitability(sess, ctypes.byref(expl), ctypes.byref(nash), None, None, None)
    exploit = expl.value if erc == 0 else None
    total_ms = ev0.elapsed_time(ev_end)
    times = [evs[i].elapsed_time(evs[i + 1]) for i in range(args.steps)]
    total_ms_max = dist_max(total_ms)
    solves = dist_sum(args.steps)
    value = solves / (total_ms_max / 1000.0)

    # end to end through ss_solve_gpu with host buffers
    out = ssg.SSOutput()
    stats = ssg.SSSolveStats()
    e2e_opts = ssg.SSSolveOptions(local, 10, -1.0, 50, 0)

    def e2e_step():
        r = lib.ss_solve_gpu_ex(ctypes.byref(sg.td), args.iterations, ctypes.byref(e2e_opts),
                                ctypes.byref(out), ctypes.byref(stats))
        check(r, "ss_solve_gpu")
        lib.ss_free_output(ctypes.byref(out))

    e2e_step()
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    torch.cuda.synchronize()
    e2e_s = dist_max(time.perf_counter() - t0)
    e2e_value = dist_sum(args.steps) / e2e_s

    np_ = cfg["num_players"]
    nh = [len(h) for h in cfg["hands"]]
    mh = max(nh)
    ndec, nnodes = sg.td.num_decision_nodes, sg.td.num_nodes
    h2d = (nnodes * 104 + sg.td.num_children_total * 4 + np_ * mh * 8 + np_ * mh * 4
           + sg.num_leaves * np_ * mh * 4)
    d2h = ndec * 8 * mh * 4 + sum(nh) * 4 + np_ * mh * 4

    dom = max((k for k in classes if k != "other"), key=lambda k: classes[k]["ms"])
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    peak = peaks.get("hbm_gbs")
    peak_src = "measured" if peak else "fallback"
    if not peak:
        peak = 6650.0
    d = classes[dom]
    # per launch: algorithmic bytes and average event-timed duration (their
    # ratio equals bytes per iteration over time per iteration)
    n_launch = max(1, d["launches"])
    achieved = d["bytes"] / (d["ms"] / 1e3) / 1e9 if d["ms"] > 0 else 0.0
    traffic, traffic_note = None, "no ncu capture of this workload"
    try:
        tr = json.load(open(os.path.join(ROOT, "profiles", "dram_traffic.json")))
        if tr.get("kernel_sources_sha16") != kernel_sources_sha16():
            traffic_note = "the ncu capture predates the current kernel sources"
        else:
            tcls = tr.get("workloads", {}).get(args.workload, {}).get("classes", {})
            if dom in tcls:
                traffic = tcls[dom].get("dram_bytes_per_launch")
                traffic_note = tr.get("source", "")
    except Exception:
        pass

    tree_info = {"nodes": nnodes, "decision": ndec, "leaves": sg.num_leaves, "hands": nh}
    # whole iterations against the bytes the reference's own data flow moves
    # per iteration on this tree (formula in flow_bytes_per_iteration)
    flow = flow_bytes_per_iteration(sg.td, mh)
    t_iter = (total_ms_max / args.steps) / args.iterations / 1e3   # seconds, uninstrumented
    flow_gbs = flow / t_iter / 1e9
    roof_iter = {"bytes_per_iteration": flow, "iteration_ms": t_iter * 1e3, "achieved": flow_gbs, "peak": peak,
                 "peak_source": peak_src, "unit": "GB/s", "frac": flow_gbs / peak,
                 "basis": "reference data flow per iteration: regret matching of every decision node, "
                          "reach of every non-traverser player, values, terminals (per traverser)"}
    lib.ss_session_destroy(sess)
    sg.free()
    return {
        "value": value, "ms_per_step": total_ms_max / args.steps, "times": times,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h)},
        "clocks": clk,
        "gpu_launches": int(args.steps * (args.iterations * launches_per_iter + reach_launches)),
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                     "peak_source": peak_src, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "traffic_source": traffic_note,
                     "bytes_per_launch": d["bytes"] / n_launch,
                     "launch_ms": d["ms"] / n_launch, "launches_per_iteration": d["launches"],
                     "bytes_per_iteration": d["bytes"], "kernel_ms_per_iteration": d["ms"]},
        "profile": {k: {"ms": round(v["ms"], 4), "launches": v["launches"],
                        "GBps": round(v["bytes"] / (v["ms"] / 1e3) / 1e9, 1) if v["ms"] > 0 else 0}
                    for k, v in classes.items() if v["launches"]},
        "iteration_ms": prof.iteration_ms,
        "profile_launches": launch_list,
        "exploitability_pct": exploit,
        "tree": tree_info,
        "roofline_iteration": roof_iter,
        # node-hand updates: nodes x sum of the players' hand counts, per iteration
        "nhu_per_solve": float(nnodes) * sum(nh) * args.iterations,
    }


# ---------------------------------------------------------------------------
# batched and served forms on the request mix
# ---------------------------------------------------------------------------

TARGET = 0.5      # % of pot
CHECK = 25        # iterations between exploitability checks
MAX_ITERS = 1000


def pct(v, q):
    v = sorted(v)
    return v[min(len(v) - 1, int(round(q / 100.0 * (len(v) - 1))))]


C4_STREETS = (1 / 3, 1 / 3, 1 / 3)     # flop, turn, river
C5_STREETS = (0.05, 0.15, 0.80)
C4_MIX = ("flop / turn / river equally, 2-6 players (flops 2-3, turns 2-4), target tree size log-uniform "
          "in [50, 20000] nodes by bet-set / raise-cap search (5-6 players: trees up to 3000 nodes), 2-3 "
          "players on every combo, 4 players on 64-128 hands, 5 on 6, 6 on 4, U(0, 0.7) of each range zeroed")


def mix_stats(subs):
    nodes = [sg.td.num_nodes for sg in subs]
    kinds = {}
    for sg in subs:
        kinds[sg.cfg["name"]] = kinds.get(sg.cfg["name"], 0) + 1
    return {"tree_nodes": {"min": min(nodes), "p50": pct(nodes, 50), "max": max(nodes)}, "kinds": kinds}


def run_batched(n, seed, device):
    """n requests of the batched mix solved to <= 0.5% pot exploitability:
    one per call (plain form, ss_solve_gpu_ex with the same stopping rule)
    and all together (ss_batch_solve); wall time from host buffers to host
    outputs for both."""
    import workloads as wl
    subs = wl.c4_subgames(n, seed, streets=C4_STREETS)
    sg0 = subs[0]
    rc, _ = sg0.solve(CHECK, target=TARGET, check_every=CHECK)  # warm the library / pool
    t0 = time.perf_counter()
    plain, by_kind = [], {}
    for sg in subs:
        t1 = time.perf_counter()
        rc, r = sg.solve(MAX_ITERS, target=TARGET, check_every=CHECK, device=device)
        if rc != 0:
            raise RuntimeError(f"plain solve failed ({rc}): {wl.ssg.last_error(sg.lib)}")
        plain.append(r["stats"])
        k = by_kind.setdefault(sg.cfg["name"], {"n": 0, "s": 0.0, "iterations": 0, "max_ms": 0.0})
        dt = time.perf_counter() - t1
        k["n"] += 1
        k["s"] += dt
        k["iterations"] += r["stats"]["iterations_run"]
        k["max_ms"] = max(k["max_ms"], dt * 1e3)
    t_plain = time.perf_counter() - t0
    # warm the batched path (its kernels load on first use) as the plain
    # leg was warmed above: one short batch over the first requests
    rc, _ = wl.batch_solve(subs[:16], CHECK, target=TARGET, check_every=CHECK, device=device)
    t0 = time.perf_counter()
    rc, res = wl.batch_solve(subs, MAX_ITERS, target=TARGET, check_every=CHECK, device=device)
    t_batch = time.perf_counter() - t0
    if rc != 0:
        raise RuntimeError(f"batch solve failed ({rc}): {wl.ssg.last_error(sg0.lib)}")
    its = [r["stats"]["iterations_run"] for r in res]
    expl = [r["stats"]["exploitability_pct"] for r in res]
    per_it = [float(sg.td.num_nodes) * float(sum(sg.nh)) for sg in subs]   # node-hand updates per iteration
    nhu_batch = sum(n_ * k for n_, k in zip(per_it, its))
    nhu_plain = sum(n_ * p["iterations_run"] for n_, p in zip(per_it, plain))
    gpu_ms = res[0]["stats"]["solve_ms"]
    mix = mix_stats(subs)
    for sg in subs:
        sg.free()
    out = {"subgames": n, "target_pct": TARGET, "check_every": CHECK,
           "plain_solves_per_s": n / t_plain, "batched_solves_per_s": n / t_batch,
           "speedup_vs_plain": t_plain / t_batch,
           "plain_node_hand_updates_per_s": nhu_plain / t_plain,
           "batched_node_hand_updates_per_s": nhu_batch / t_batch,
           "batched_wall_s": t_batch, "batched_gpu_iterations_s": gpu_ms / 1e3,
           "plain_wall_s": t_plain,
           "iterations_p50": pct(its, 50), "iterations_max": max(its),
           "exploitability_max_pct": max(expl),
           "plain_iterations_p50": pct([p["iterations_run"] for p in plain], 50),
           # where the plain form's time goes: per request kind, requests,
           # summed solve seconds, iterations run, slowest solve
           "plain_by_kind": {k: {"n": v["n"], "s": round(v["s"], 3), "iterations": v["iterations"],
                                 "max_ms": round(v["max_ms"], 1)} for k, v in sorted(by_kind.items())},
           "mix": C4_MIX}
    out.update(mix)
    return out


def run_served(rates, n, seed, device):
    """Poisson arrivals of n requests of the served mix (80% river, 15% turn,
    5% flop) at each rate into the server (continuous batching, retirement at
    <= 0.5% pot); latency = submission to retirement.  The plain form's
    service time of the same requests (one solve per call, no queueing) is
    reported beside it."""
    import workloads as wl
    subs = wl.c4_subgames(n, seed + 1, streets=C5_STREETS)
    lib = subs[0].lib
    per_rate = []
    for rate in rates:
        rng = np.random.default_rng(seed + 7)
        gaps = rng.exponential(1.0 / rate, n)
        srv = wl.Server(lib, device=device, block_iterations=CHECK, target_exploitability=TARGET,
                        max_iterations=MAX_ITERS, memory_budget_gb=60.0)
        ids = [None] * n
        t_start = time.perf_counter()

        def feeder():
            t = t_start
            for i, sg in enumerate(subs):
                t += gaps[i]
                d = t - time.perf_counter()
                if d > 0:
                    time.sleep(d)
                ids[i] = srv.submit(sg)

        th = threading.Thread(target=feeder)
        th.start()
        lat, queue, its, nhu = [], [], [], []
        for i, sg in enumerate(subs):
            while ids[i] is None:
                time.sleep(0.0005)
            r = srv.wait(ids[i], sg.nh)
            lat.append(r["latency_ms"])
            queue.append(r["stats"]["queue_ms"])
            its.append(r["stats"]["iterations_run"])
            nhu.append(float(sg.td.num_nodes) * float(sum(sg.nh)) * r["stats"]["iterations_run"])
        th.join()
        wall = time.perf_counter() - t_start
        srv.close()
        per_rate.append({"rate_per_s": rate, "requests": n, "arrivals_s": float(gaps.sum()),
                         "solves_per_s": n / wall, "node_hand_updates_per_s": sum(nhu) / wall,
                         "latency_p50_ms": pct(lat, 50), "latency_p99_ms": pct(lat, 99),
                         # latency = queueing (submission until the request joins
                         # the running batch) + time in the batch
                         "queue_p50_ms": pct(queue, 50), "queue_p99_ms": pct(queue, 99),
                         "in_batch_p50_ms": pct([a - b for a, b in zip(lat, queue)], 50),
                         "in_batch_p99_ms": pct([a - b for a, b in zip(lat, queue)], 99),
                         "offered_over_served": rate / (n / wall),
                         "iterations_p50": pct(its, 50)})
    service = []
    for sg in subs[:min(n, 64)]:
        t0 = time.perf_counter()
        rc, _ = sg.solve(MAX_ITERS, target=TARGET, check_every=CHECK, device=device)
        service.append((time.perf_counter() - t0) * 1e3)
    out = {"rates": per_rate,
           "plain_service_p50_ms": pct(service, 50), "plain_service_p99_ms": pct(service, 99),
           "plain_solves_per_s": 1e3 * len(service) / sum(service),
           "mix": "the batched mix with streets 5% flop / 15% turn / 80% river"}
    out.update(mix_stats(subs))
    for sg in subs:
        sg.free()
    return out


# ---------------------------------------------------------------------------
# the reference on the host cores
# ---------------------------------------------------------------------------

class _Quiet:
    """Silence the reference's printf progress lines (fd 1) during a call."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        self.null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self.null, 1)

    def __exit__(self, *a):
        os.dup2(self.saved, 1)
        os.close(self.saved)
        os.close(self.null)


def run_leaf_producer(seed, calls=3):
    """Continuation values of the 3-player turn subgame (the input its
    15,616 continuation leaves read) produced through the host module
    leaf_values.compute_turn_leaf_values -> ss_leaf_values_gpu: host plan,
    upload, kernels and the 126 MB of values copied back, wall clock per
    call.  Beside it the oracle's loop form of the reference's Python
    producer (python/leaf_values.py:694-816) on a bounded sample: 100 hero
    hands of one (river card, player) pair and 100,000 bias-adjusted values,
    scaled to 12 river cards x 3 players x 1128 hands and every value."""
    import leaf_values as lv
    import workloads as wl
    from oracle import leaf_oracle
    from oracle.oracle import Oracle
    cfg = wl.config("turn3", seed=seed)
    sg = wl.AbiSubgame(cfg)
    try:
        infos = lv.extract_leaf_info_from_tree(sg.td, cfg["num_players"])
    finally:
        sg.free()
    N = cfg["num_players"]
    ph = [[(int(h[0]), int(h[1]), float(w)) for h, w in zip(cfg["hands"][p], cfg["weights"][p])] for p in range(N)]
    mh = max(len(h) for h in ph)
    lv.compute_turn_leaf_values(cfg["board"], infos, mh, cfg["pot"], player_hands=ph)   # warm-up
    times = []
    for _ in range(calls):
        t0 = time.perf_counter()
        out = lv.compute_turn_leaf_values(cfg["board"], infos, mh, cfg["pot"], player_hands=ph)
        times.append((time.perf_counter() - t0) * 1e3)
    runouts = lv.turn_runouts(cfg["board"], [len(h) for h in ph])
    orc = Oracle()
    b5 = list(cfg["board"]) + runouts[0]
    strength = [{h: orc.eval7(b5 + [c0, c1]) for h, (c0, c1, _w) in enumerate(ph[p])
                 if c0 not in b5 and c1 not in b5} for p in range(N)]
    sample_hands = 100
    strength[0] = dict(list(strength[0].items())[:sample_hands])
    raw = np.zeros((N, mh))
    cnt = np.zeros((N, mh))
    t0 = time.perf_counter()
    leaf_oracle._equity_one_runout(0, ph, strength, raw, cnt)
    eq_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    for k in range(100000):
        leaf_oracle.biased_value(0.25, 300, k & 3, (k >> 2) & 3)
    bias_s = time.perf_counter() - t0
    cpu_ms = 1e3 * (eq_s * len(runouts) * N * mh / sample_hands + bias_s * out.size / 100000)
    t = sorted(times)
    return {"workload": f"3-player turn subgame leaf values: {len(infos)} leaf descriptors x 64 profiles x "
                        f"{N} players x {mh} hands ({out.nbytes / 1e6:.0f} MB FP32), {len(runouts)} river cards, "
                        f"2000 sampled opponent pairs per (river, player)",
            "ms_per_call_e2e": t[len(t) // 2], "calls": calls, "d2h_bytes_per_call": int(out.nbytes),
            "cpu_baseline": {"ms_per_call": cpu_ms, "cores": 1, "kind": "port",
                             "sample": f"oracle loop form of python/leaf_values.py: {sample_hands} hero hands of "
                                       f"one (river, player) pair ({eq_s:.2f} s) and 100,000 bias values "
                                       f"({bias_s:.2f} s), scaled"}}


def session_iteration_profile(lib, td, device, reps=3, warm=2):
    """Device time of one CFR iteration of a resident session (CUDA events
    between kernel classes, ss_session_profile): `warm` plain iterations,
    then `reps` profiled ones; returns the median iteration and, per kernel
    class, its median time."""
    import street_solver_gpu as ssg

    class Prof(ctypes.Structure):
        _fields_ = [("num_classes", ctypes.c_int), ("name", (ctypes.c_char * 16) * 8),
                    ("launches", ctypes.c_int * 8), ("ms", ctypes.c_double * 8),
                    ("bytes", ctypes.c_double * 8), ("iteration_ms", ctypes.c_double)]

    lib.ss_session_destroy.argtypes = [ctypes.c_void_p]
    lib.ss_session_run.argtypes = [ctypes.c_void_p, ctypes.c_int]
    opts = ssg.SSSolveOptions(device, 10, -1.0, 50, 0)
    sess = ctypes.c_void_p()
    rc = lib.ss_session_create(ctypes.byref(td), ctypes.byref(opts), ctypes.byref(sess))
    if rc != 0:
        raise RuntimeError(f"ss_session_create failed ({rc}): {ssg.last_error(lib)}")
    try:
        if warm:
            rc = lib.ss_session_run(sess, warm)
            if rc != 0:
                raise RuntimeError(f"ss_session_run failed ({rc}): {ssg.last_error(lib)}")
        its, cls = [], {}
        for _ in range(reps):
            prof = Prof()
            rc = lib.ss_session_profile(sess, ctypes.byref(prof))
            if rc != 0:
                raise RuntimeError(f"ss_session_profile failed ({rc}): {ssg.last_error(lib)}")
            its.append(prof.iteration_ms)
            for k in range(prof.num_classes):
                if prof.launches[k]:
                    name = bytes(prof.name[k]).split(b"\0")[0].decode()
                    cls.setdefault(name, []).append(prof.ms[k])
    finally:
        lib.ss_session_destroy(sess)
    med = lambda v: sorted(v)[len(v) // 2]
    return med(its), {k: round(med(v), 3) for k, v in cls.items()}


def run_four_player(seed, device, reps=3):
    """4-player subgames with full ranges, whose terminals with three counted
    opponents take the closed forms (folds and leaves: k_term_cr3, four-way
    showdowns: k_term_sd3): a turn with continuation leaves (1128 combos per
    player, U(0,1) weights with 30% zeroed, pot 150, stacks 500, bets {1.0
    pot} + all-in, one raise, leaf values N(0, 0.3 pot); 5,681 nodes) and a
    river (1081 combos per player, U(0,1) weights, pot 300, stacks 1000, the
    same bets; 125 nodes).  Device time per iteration: the median of `reps`
    profiled iterations of a resident session (after two plain ones), with
    the per-kernel-class split."""
    import workloads as wl
    out = {}
    for street, name in (("turn", "turn3"), ("river", "river6")):
        cfg = wl.config(name, seed=seed, num_players=4, bet_sizes=[1.0], max_raises=1)
        cfg["hands"], cfg["weights"] = wl.make_ranges(np.random.default_rng(seed + 4), cfg["board"], 4, None,
                                                      zero_frac=0.3 if street == "turn" else 0.0)
        sg = wl.AbiSubgame(cfg)
        try:
            sg.set_leaf_values(wl.leaf_values_for(cfg, sg.num_leaves))
            it_ms, classes = session_iteration_profile(sg.lib, sg.td, device, reps=reps)
            nodes, nh = sg.td.num_nodes, [len(h) for h in cfg["hands"]]
        finally:
            sg.free()
        per_it = it_ms / 1e3
        out[street] = {"tree_nodes": nodes, "hands": nh[0], "ms_per_iteration": it_ms, "classes_ms": classes,
                       "node_hand_updates_per_s": nodes * sum(nh) / per_it if per_it > 0 else None,
                       "solve_1000_iterations_s_est": 1000 * per_it}
    out["sample"] = f"median of {reps} profiled iterations (CUDA events per kernel class) after 2 plain ones"
    return out


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def run_hu_river(seed, device, solves=5, cpu_iterations=20):
    """The heads-up river configuration, the reference's CPU-runnable case:
    5-card board, both ranges all 1081 combos with U(0,1) weights, pot 100,
    stacks 400, bets {0.5, 1.0 pot} + all-in, 2 raises, 1000 Linear-CFR
    iterations.  GPU: ss_solve_gpu_ex from host buffers to host outputs, wall
    clock per solve after one warm-up solve.  CPU: the reference's own CPU
    solver src/solver.c (-O2 -fopenmp, single-threaded per solve), one solve
    per host core at once (one OS thread each), timed on cpu_iterations
    iterations and scaled to 1000; its rules differ from street_solve.cu's
    (a timing baseline, not a parity target)."""
    import workloads as wl
    cfg = wl.config("hu_river", seed=seed)
    iters = cfg["iterations"]
    sg = wl.AbiSubgame(cfg)
    try:
        rc, _ = sg.solve(iters, device=device)
        if rc != 0:
            raise RuntimeError(f"ss_solve_gpu failed ({rc})")
        times = []
        for _ in range(solves):
            t0 = time.perf_counter()
            rc, _ = sg.solve(iters, device=device)
            times.append(time.perf_counter() - t0)
            if rc != 0:
                raise RuntimeError(f"ss_solve_gpu failed ({rc})")
        nodes = sg.td.num_nodes
    finally:
        sg.free()
    t = sorted(times)
    out = {"workload": "heads-up river, 1081 combos per player, 2 raises, 1000 iterations",
           "tree_nodes": nodes, "gpu_ms_per_solve_e2e": 1e3 * t[len(t) // 2],
           "gpu_solves_per_s": len(times) / sum(times), "cpu_baseline": None}
    try:
        from oracle.oracle import RefSolverC, ref_solver_available
    except ImportError:
        return out
    if not ref_solver_available():
        return out
    ref = RefSolverC()
    cores = os.cpu_count() or 1
    secs = [None] * cores

    def one(i):
        secs[i] = ref.solve(cfg["board"], cfg["hands"], cfg["weights"], cfg["pot"], cfg["stack"],
                            cfg["bet_sizes"], cpu_iterations)

    with _Quiet():
        th = [threading.Thread(target=one, args=(i,)) for i in range(cores)]
        t0 = time.perf_counter()
        for x in th:
            x.start()
        for x in th:
            x.join()
        wall = time.perf_counter() - t0
    scale = iters / cpu_iterations
    per_solve = statistics.median(secs) * scale
    out["cpu_baseline"] = {"solves_per_s": cores / (wall * scale), "s_per_solve": per_solve, "cores": cores,
                           "cpu_model": cpu_model(), "kind": "reference",
                           "sample": f"src/solver.c, {cores} concurrent solves of {cpu_iterations} iterations "
                                     f"({wall:.1f} s wall), scaled to {iters}"}
    return out


def reference_cpu(seed, budget_s=25.0):
    """Seconds per CFR iteration of the reference kernels (host build) on the
    full turn3 tree, measured at small range sizes with every core running
    its own solve, and extrapolated to 1128 hands per player."""
    import workloads as wl
    from oracle.oracle import RefStreetSolve, ref_available
    if not ref_available(200, 3):
        return None
    ref = RefStreetSolve(200, 3, "cpu")
    cores = os.cpu_count() or 1
    full = wl.config(WORKLOAD, seed=seed)
    sizes, per_iter = [], []
    t_start = time.perf_counter()
    # the two-opponent terminals enumerate opponent pairs per hand (cost ~H^3
    # once per-node overhead stops dominating): the fit uses the two largest
    # sizes that fit the time budget
    for H in (8, 12, 16, 24):
        cfg = wl.config(WORKLOAD, seed=seed, num_hands=H)
        Hm, Wm, nh = wl.padded(cfg)
        results = [None] * cores

        def one(i):
            td = ref.build(cfg["board"], cfg["pot"], cfg["stack"], cfg["bet_sizes"], 3)
            lv = wl.leaf_values_for(cfg, td.num_leaves)
            t0 = time.perf_counter()
            ref.solve(td, Hm, Wm, nh, 1, leaf_values=lv)
            results[i] = time.perf_counter() - t0
            ref.free(td)

        with _Quiet():
            th = [threading.Thread(target=one, args=(i,)) for i in range(cores)]
            t0 = time.perf_counter()
            for t in th:
                t.start()
            for t in th:
                t.join()
            wall = time.perf_counter() - t0
        sizes.append(H)
        per_iter.append(wall / cores)  # aggregate seconds per iteration per solve
        if time.perf_counter() - t_start > budget_s:
            break
    x, y = np.log(np.array(sizes[-2:], float)), np.log(np.array(per_iter[-2:], float))
    expo = float((y[1] - y[0]) / (x[1] - x[0])) if len(sizes) >= 2 else 3.0
    H_full = len(full["hands"][0])
    s_iter_full = per_iter[-1] * (H_full / sizes[-1]) ** expo
    return {"cores": cores, "sizes": sizes, "sec_per_iter": per_iter, "exponent": expo,
            "sec_per_iter_full": s_iter_full,
            "solves_per_s": 1.0 / (s_iter_full * 1000)}


FLOP = {"flop": [0, 13, 26], "pot": 1000, "stack": 5000, "bet_sizes": [0.75], "hands": 200, "iterations": 100}


def run_flop(seed, device, solves=3):
    """The multi-street (flop through river) solver against the reference's
    own sm_100a build of src/cuda/flop_solve.cu on the same tree, ranges and
    iterations, both through fs_solve_gpu from host buffers on this GPU:
    median wall time per solve."""
    import flop_solve as fsm
    import street_solver_gpu as ssg
    import workloads as wl
    ref_path = os.path.join(ROOT, "oracle", "_ref", "libref_flop_solve_gpu.so")
    rng = np.random.default_rng(seed + 11)
    h, w = wl.make_ranges(rng, FLOP["flop"], 2, FLOP["hands"])
    out = {"workload": f"flop-through-river 2 players, flop {FLOP['flop']}, pot {FLOP['pot']}, stack {FLOP['stack']}, "
                       f"flop bets {FLOP['bet_sizes']} (turn / river 0.75), {FLOP['hands']} hands each, "
                       f"{FLOP['iterations']} Linear-CFR iterations"}
    libs = [("ours", ssg.load_library(200))]
    if os.path.exists(ref_path):
        libs.append(("reference_gpu", ctypes.CDLL(ref_path)))
    for name, lib in libs:
        sg = fsm.FlopSubgame(lib, FLOP["flop"], FLOP["pot"], FLOP["stack"], FLOP["bet_sizes"], h, w)
        out["tree_nodes"] = sg.td.num_nodes
        times = []
        with _Quiet():
            for _ in range(solves + 1):
                t0 = time.perf_counter()
                sg.solve(FLOP["iterations"])
                times.append(time.perf_counter() - t0)
        sg.free()
        times = sorted(times[1:])
        out[name + "_s_per_solve"] = times[len(times) // 2]
    if "reference_gpu_s_per_solve" in out:
        out["speedup_vs_reference_gpu"] = out["reference_gpu_s_per_solve"] / out["ours_s_per_solve"]
    return out


ANCHOR = {"hands": 10, "iterations": 20}


def anchor_config(seed):
    import workloads as wl
    cfg = wl.config(WORKLOAD, seed=seed, num_hands=ANCHOR["hands"])
    return cfg, (f"3-player turn subgame with continuation leaves, the benchmark's 21,436-node tree, "
                 f"{ANCHOR['hands']} combos/player, {ANCHOR['iterations']} Linear-CFR iterations")


def anchor_reference(seed):
    """The same small configuration solved by the reference's kernels on the
    host (oracle/_ref), one solve per core at once: measured, not modelled."""
    import workloads as wl
    from oracle.oracle import RefStreetSolve, ref_available
    if not ref_available(200, 3):
        return None
    ref = RefStreetSolve(200, 3, "cpu")
    cores = os.cpu_count() or 1
    cfg, name = anchor_config(seed)
    Hm, Wm, nh = wl.padded(cfg)

    def one(i):
        td = ref.build(cfg["board"], cfg["pot"], cfg["stack"], cfg["bet_sizes"], 3)
        lv = wl.leaf_values_for(cfg, td.num_leaves)
        ref.solve(td, Hm, Wm, nh, ANCHOR["iterations"], leaf_values=lv)
        ref.free(td)

    with _Quiet():
        th = [threading.Thread(target=one, args=(i,)) for i in range(cores)]
        t0 = time.perf_counter()
        for t in th:
            t.start()
        for t in th:
            t.join()
        wall = time.perf_counter() - t0
    return {"workload": name, "solves_per_s": cores / wall, "wall_s": wall, "solves": cores, "cores": cores,
            "kind": "reference kernels on the host (oracle/_ref), one solve per core"}


def anchor_gpu(seed, device, solves=20):
    """The same small configuration through ss_solve_gpu from host buffers."""
    import workloads as wl
    cfg, name = anchor_config(seed)
    sg = wl.AbiSubgame(cfg, max_hands=200)
    sg.set_leaf_values(wl.leaf_values_for(cfg, sg.num_leaves))
    rc, _ = sg.solve(ANCHOR["iterations"], device=device)   # warm
    t0 = time.perf_counter()
    for _ in range(solves):
        rc, _ = sg.solve(ANCHOR["iterations"], device=device)
        if rc != 0:
            raise RuntimeError(f"anchor solve failed ({rc})")
    wall = time.perf_counter() - t0
    sg.free()
    return {"workload": name, "solves_per_s": solves / wall, "wall_s": wall, "solves": solves,
            "kind": "ss_solve_gpu from host buffers (e2e), one B200"}


def main():
    args = parse()
    if args.ncu_summary:
        tr = ncu_summary(args.ncu_summary[0], args.workload, args.ncu_summary[1])
        print(json.dumps(tr["workloads"][args.workload]))
        return 0
    world, rank, local = dist_init()
    if args.impl == "reference":
        if rank == 0:
            # one bounded sample per step (the extrapolated full-size rate);
            # the line reports their median
            runs = [reference_cpu(args.seed) for _ in range(max(1, args.steps))]
            r = None if any(x is None for x in runs) else dict(
                sorted(runs, key=lambda x: x["solves_per_s"])[len(runs) // 2],
                samples=[x["solves_per_s"] for x in runs])
            if r is None:
                print(json.dumps({"impl": "reference",
                                  "unavailable": "oracle/_ref reference build missing"}))
            else:
                line = {
                    "impl": "reference", "metric": METRIC, "value": r["solves_per_s"], "unit": UNIT,
                    "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                    "ms_per_step": 1000.0 / r["solves_per_s"], "higher_is_better": True,
                    "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                    "config": {"workload": "3-player turn subgame, 1128 combos/player, "
                                           "continuation leaves, 1000 Linear-CFR iterations",
                               "iterations": args.iterations},
                    "cpu_baseline": {"value": r["solves_per_s"], "unit": UNIT, "cores": r["cores"],
                                     "kind": "reference",
                                     "sample": f"street_solve.cu kernels on the host, full 21,436-node "
                                               f"tree, 1 iteration at {r['sizes']} hands/player, "
                                               f"extrapolated to 1128 with exponent "
                                               f"{r['exponent']:.2f}; median of {len(r['samples'])} samples"},
                    "samples": r["samples"],
                    "value_is_model": "full-size rate extrapolated from measured small-range iterations "
                                      "(the reference's O(H^3) terminals cannot run 1128 hands in bounded "
                                      "time); anchor_same_config is measured on a config both arms run",
                    "anchor_same_config": anchor_reference(args.seed),
                    "e2e": {"value": r["solves_per_s"], "unit": UNIT, "h2d_bytes_per_step": 0,
                            "d2h_bytes_per_step": 0},
                }
                print(json.dumps(line))
        return 0

    forms = set(args.forms.split(","))
    res = run_ours(args, world, rank, local)
    batched = served = None
    if rank == 0 and world == 1 and "batched" in forms:
        try:
            batched = run_batched(args.batch_size, args.seed, local)
        except Exception as e:  # the solver's line is printed whatever happens here
            batched = {"error": f"{type(e).__name__}: {e}"}
    if rank == 0 and world == 1 and "served" in forms:
        try:
            served = run_served([float(r) for r in args.rates.split(",")], args.served_requests, args.seed, local)
        except Exception as e:  # the solver's line is printed whatever happens here
            served = {"error": f"{type(e).__name__}: {e}"}
    hu = None
    if rank == 0 and world == 1 and "hu_river" in forms:
        try:
            hu = run_hu_river(args.seed, local)
        except Exception as e:  # the solver's line is printed whatever happens here
            hu = {"error": f"{type(e).__name__}: {e}"}
    leaf = None
    if rank == 0 and world == 1 and "leaf" in forms and args.workload == "turn3":
        try:
            leaf = run_leaf_producer(args.seed)
        except Exception as e:  # the solver's line is printed whatever happens here
            leaf = {"error": f"{type(e).__name__}: {e}"}
    four = None
    if rank == 0 and world == 1 and "four" in forms:
        try:
            four = run_four_player(args.seed, local)
        except Exception as e:  # the solver's line is printed whatever happens here
            four = {"error": f"{type(e).__name__}: {e}"}
    flop = None
    if rank == 0 and world == 1 and "flop" in forms:
        try:
            flop = run_flop(args.seed, local)
        except Exception as e:  # the solver's line is printed whatever happens here
            flop = {"error": f"{type(e).__name__}: {e}"}
    anchor = None
    if rank == 0 and world == 1 and "anchor" in forms and args.workload == "turn3":
        try:
            anchor = {"gpu": anchor_gpu(args.seed, local), "reference": anchor_reference(args.seed)}
            if anchor["reference"]:
                anchor["speedup"] = anchor["gpu"]["solves_per_s"] / anchor["reference"]["solves_per_s"]
        except Exception as e:  # the solver's line is printed whatever happens here
            anchor = {"error": f"{type(e).__name__}: {e}"}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and args.workload == "turn3":
        r = reference_cpu(args.seed, budget_s=20.0)
        if r is not None:
            cpu = {"value": r["solves_per_s"], "unit": UNIT, "cores": r["cores"], "kind": "reference",
                   "sample": f"street_solve.cu kernels on the host, full tree, 1 iteration at "
                             f"{r['sizes']} hands/player, extrapolated to 1128 (exponent "
                             f"{r['exponent']:.2f})"}
    if rank == 0:
        t = sorted(res["times"])
        line = {
            "metric": METRIC, "value": res["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": res["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOADS[args.workload][0],
                       "iterations": args.iterations, "tree": res["tree"],
                       "l2": WORKLOADS[args.workload][1],
                       "parallelism": f"replicas x{world}",
                       "p50_ms": t[len(t) // 2], "p99_ms": t[-1]},
            "roofline": res["roofline"], "roofline_iteration": res["roofline_iteration"],
            "cpu_baseline": cpu, "clocks": res["clocks"],
            "e2e": res["e2e"], "gpu_launches": res["gpu_launches"],
            "node_hand_updates_per_s": res["value"] * res["nhu_per_solve"],
            "iteration_ms": res["iteration_ms"], "profile": res["profile"],
            "profile_launches": res["profile_launches"],
            "exploitability_pct_after_solve": res["exploitability_pct"],
            "batched": batched, "served": served, "hu_river": hu, "leaf_producer": leaf, "four_player": four,
            "anchor_same_config": anchor, "flop_solver": flop,
            "hu_river_vs_reference_cpu": None if not hu or "error" in hu else {
                "gpu_solves_per_s": hu.get("gpu_solves_per_s"),
                "reference_cpu_solves_per_s": (hu.get("cpu_baseline") or {}).get("solves_per_s")},
        }
        print(json.dumps(line))
    try:
        import torch.distributed as dist
        if dist.is_initialized():
            dist.destroy_process_group()
    except Exception:
        pass
    return 0


if __name__ == "__main__":
    sys.exit(main())
