"""Host-side check of the planner's three-way showdown sweep tables
(ss_plan.cpp): the per-player segments tile the rank axis, a segment holding
the player's hands is one tie group, the runs cover the segments in order
with about equal cost and at most one wave of blocks per traverser, and the
planned spans bound every run (and every merged group of runs) that a
kernel block carves class storage for.  The planner and tree builder are
compiled with g++ into a small driver (tests/native/plan_runs.cpp)."""
import json
import os
import shutil
import subprocess

import pytest

from cards import card_to_int

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "poker-solver_b200", "csrc")


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    out = str(tmp_path_factory.mktemp("plan") / "plan_runs")
    subprocess.run(["g++", "-O1", "-std=c++17", "-I", os.path.join(ROOT, "include"), "-I", CSRC,
                    os.path.join(ROOT, "tests", "native", "plan_runs.cpp"), os.path.join(CSRC, "ss_plan.cpp"),
                    os.path.join(CSRC, "ss_tree.cpp"), "-o", out], check=True)
    return out


def plan(driver, seed, hands, board):
    cards = [str(card_to_int(c)) for c in board]
    r = subprocess.run([driver, str(seed), str(hands)] + cards, check=True, capture_output=True, text=True)
    return json.loads(r.stdout)


CASES = [
    (0, 1081, ["2c", "7d", "9h", "Js", "Kc"]),
    (1, 1081, ["As", "Ad", "5c", "5h", "Tc"]),
    (2, 400, ["3s", "8s", "Qs", "4d", "6h"]),
    (3, 60, ["2h", "3d", "9c", "Tc", "Jd"]),
    (4, 1081, ["Ts", "Js", "Qs", "Ks", "As"]),     # every combo ties: one group
    (5, 1081, ["Kc", "Kd", "Kh", "Ks", "2c"]),     # quads on board
]


@pytest.mark.parametrize("seed,hands,board", CASES)
def test_sweep_runs(driver, seed, hands, board):
    d = plan(driver, seed, hands, board)
    nc, K16 = d["ncomb"], d["chunks"]
    spans = [0] * len(d["spans"])
    for p in d["players"]:
        assert p["flags_ok"]
        segs, base, ch = p["segs"], p["seg_base"], p["chunk"]
        # segments tile [0, ncomb) in rank order
        assert segs[0][0] == 0 and segs[-1][1] == nc
        assert all(segs[i][1] == segs[i + 1][0] for i in range(len(segs) - 1))
        assert all(lo < hi for lo, hi, _ in segs)
        # runs: in order, covering every segment once, the used ones first
        assert ch[0] == base and ch[-1] == base + len(segs) and len(ch) == K16 + 1
        assert all(ch[k] <= ch[k + 1] for k in range(K16))
        used = [k for k in range(K16) if ch[k + 1] > ch[k]]
        K = len(used)
        assert used == list(range(K))
        nt = p["sd2_terminals"]
        if nt:
            assert K <= max(1, d["slots"] // nt)
        # about equal cost: a run ends at the first segment boundary reaching
        # its share, so it exceeds the share by less than one segment
        cost = [d["seg_cost"] + hi - lo for lo, hi, _ in segs]
        total = sum(cost)
        for k in used[:-1]:
            run = sum(cost[ch[k] - base:ch[k + 1] - base])
            assert run < total / K + max(cost) + 1
        # spans of 2^lg merged runs
        for lg in range(len(spans)):
            m = 1 << lg
            for r in range(0, K16, m):
                s0, s1 = ch[r] - base, ch[r + m] - base
                if s1 > s0:
                    spans[lg] = max(spans[lg], segs[s1 - 1][1] - segs[s0][0])
    assert spans == d["spans"]
    assert all(spans[i] <= spans[i + 1] for i in range(len(spans) - 1)) and spans[-1] == nc


def test_one_wave_cap(driver):
    # a full-range 3-player river: 40 three-way showdowns per traverser, so
    # 592 // 40 = 14 runs although the cost alone would allow 16
    d = plan(driver, 0, 1081, CASES[0][2])
    for p in d["players"]:
        assert p["sd2_terminals"] == 40
        used = sum(1 for k in range(d["chunks"]) if p["chunk"][k + 1] > p["chunk"][k])
        assert used == 14
