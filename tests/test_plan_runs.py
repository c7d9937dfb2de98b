"""Host-side checks of the planner (ss_plan.cpp), compiled with g++ with the
tree builder into small drivers (tests/native/):
* plan_runs: the three-way showdown sweep tables -- the per-player segments
  tile the rank axis, a segment holding the player's hands is one tie group,
  the runs cover the segments in order with about equal cost and at most one
  wave of blocks per traverser, and the planned spans bound every run (and
  every merged group of runs) that a kernel block carves class storage for;
* plan_kinds: the terminal routing -- each terminal goes to the closed form
  for its number of counted opponents (folds count every other player,
  showdowns and leaves the live ones), the scatter form for ranges that
  repeat a combo, and exact enumeration for the rest."""
import json
import os
import shutil
import subprocess

import pytest

from cards import card_to_int

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "poker-solver_b200", "csrc")


def _compile(tmp_path_factory, name):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    out = str(tmp_path_factory.mktemp("plan") / name)
    subprocess.run(["g++", "-O1", "-std=c++17", "-I", os.path.join(ROOT, "include"), "-I", CSRC,
                    os.path.join(ROOT, "tests", "native", name + ".cpp"), os.path.join(CSRC, "ss_plan.cpp"),
                    os.path.join(CSRC, "ss_tree.cpp"), "-o", out], check=True)
    return out


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    return _compile(tmp_path_factory, "plan_runs")


@pytest.fixture(scope="module")
def kinds_driver(tmp_path_factory):
    return _compile(tmp_path_factory, "plan_kinds")


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


# TermKind values (ss_engine.h)
ZERO, LEAF0, CR1, CR2, SD1, ENUM, SD2, CR1D, CR3, SD3 = range(10)
FOLD, SHOWDOWN, LEAF = 1, 2, 4
CR3_MIN_HANDS = 16   # kCr3MinHands


def expected_kinds(d, np_, river, leaves):
    """The routing rule restated: folds count every other player, showdowns
    (river, traverser live) and leaves (with leaf values) the live others;
    0 / 1 / 2 counted opponents take the closed forms, one opponent whose
    range repeats a combo the scatter form, three-way showdowns with such a
    range and anything else with 3+ counted opponents exact enumeration --
    except folds and leaves with exactly three, which take the conditioning
    closed form when every counted range holds at least 16 hands and the
    first two repeat no combo, and four-way showdowns, which take theirs on
    the same condition with the traverser's range repeating no combo either."""
    want = [[0] * 10 for _ in range(np_)]
    dup = d["dup"]
    nh = d["hands"]
    for typ, leaf_idx, active in d["terminals"]:
        for t in range(np_):
            opp = [o for o in range(np_) if o != t and (typ == FOLD or active[o])]
            k = len(opp)
            kind = ZERO
            if typ == FOLD or (typ == LEAF and leaves and leaf_idx >= 0):
                cr3 = (k == 3 and not dup[opp[0]] and not dup[opp[1]]
                       and all(nh[o] >= CR3_MIN_HANDS for o in opp))
                kind = (LEAF0 if k == 0 else (CR1D if dup[opp[0]] else CR1) if k == 1
                        else CR2 if k == 2 else CR3 if cr3 else ENUM)
            elif typ == SHOWDOWN and river and active[t]:
                nodup = k >= 2 and not (dup[t] or dup[opp[0]] or dup[opp[1]])
                sd3 = k == 3 and nodup and all(nh[o] >= CR3_MIN_HANDS for o in opp)
                kind = SD1 if k == 1 else SD2 if k == 2 and nodup else SD3 if sd3 else ENUM
            want[t][kind] += 1
    return want


@pytest.mark.parametrize("np_,nb,nh,dup,leaves,raises", [
    (2, 5, 30, -1, 0, 2),     # heads-up river
    (2, 5, 30, 1, 0, 2),      # heads-up, opponent 1 repeats a combo: its folds take the scatter form
    (3, 5, 20, -1, 0, 2),     # three-way showdowns, two-opponent folds
    (3, 5, 20, 1, 0, 1),      # a repeated combo: scatter form, enumerated three-way showdowns
    (4, 5, 8, -1, 0, 1),      # three counted opponents at folds, small ranges: enumeration
    (4, 5, 20, -1, 0, 1),     # ... larger ranges: the three-opponent closed form
    (4, 5, 20, 1, 0, 1),      # ... unless a matrix opponent repeats a combo
    (4, 4, 16, -1, 1, 1),     # 4-player turn: folds and leaves with three counted opponents
    (5, 5, 20, -1, 0, 1),     # four counted opponents: enumeration
    (3, 4, 12, -1, 1, 1),     # turn with continuation leaves
    (3, 4, 12, -1, 0, 1),     # the same without leaf values: leaves are zero
])
def test_terminal_routing(kinds_driver, np_, nb, nh, dup, leaves, raises):
    r = subprocess.run([kinds_driver, str(np_), str(nb), str(nh), str(dup), str(leaves), str(raises)],
                       check=True, capture_output=True, text=True)
    d = json.loads(r.stdout)
    assert d["rc"] == 0
    assert d["dup"] == [1 if p == dup else 0 for p in range(np_)]
    assert d["kinds"] == expected_kinds(d, np_, nb == 5, leaves)
    check_groups(d)
    check_heads(d)
    inline, bad = d["cfv_inline"]
    assert bad == 0 and inline > 0, "inline value/regret frontiers decode to the frontier tables"


def check_heads(d):
    """Two-opponent launches have one block per head: every group leader
    (follow 0) that no chain head computes (chained 0), in item order; the
    one-opponent kind keeps one block per item (no heads)."""
    for t, per_kind in enumerate(d["groups"]):
        items = per_kind[1]                          # CR2
        chained = [c[1] for c in d["chains"][t]]
        want = [i for i, it in enumerate(items) if it[1] == 0 and chained[i] == 0]
        assert d["heads"][t][1] == want
        assert d["heads"][t][0] == []


def check_groups(d):
    """Closed-form terminals sharing their opponents' reach rows form
    groups: a leader with gextra followers right after it, all on the same
    rows and players, at most 16 items; nothing else shares rows with a
    neighbour outside its group."""
    for per_kind in d["groups"]:
        for items in per_kind:
            i = 0
            while i < len(items):
                lead = items[i]
                assert lead[1] == 0, "a group starts with its leader"
                n = lead[0] + 1
                assert n <= 16
                for m in items[i + 1:i + n]:
                    assert m[1] == 1 and m[2:] == lead[2:]
                nxt = items[i + n] if i + n < len(items) else None
                if nxt is not None and n < 16:
                    assert nxt[2:] != lead[2:], "a full group ends where its rows end"
                i += n



CHAIN_MAX, CHAIN_BLOCKS = 4, 2048   # kCr2ChainMax, kCr2ChainBlocks (ss_engine.h)


@pytest.mark.parametrize("raises,bets", [(2, 2), (2, 3), (3, 2), (1, 1)])
def test_two_opponent_chains(kinds_driver, raises, bets):
    """Two-opponent groups on the same first-opponent row (same opponents)
    form chains that one block computes: a head with chain = c is followed
    by c group leaders marked chained, on its first opponent's row and
    players; at most CHAIN_MAX groups per chain; followers carry no chain
    marks; and a traverser's launch keeps at least CHAIN_BLOCKS working
    blocks (small trees are not chained)."""
    r = subprocess.run([kinds_driver, "3", "4", "200", "-1", "1", str(raises), str(bets)], check=True,
                       capture_output=True, text=True)
    d = json.loads(r.stdout)
    assert d["rc"] == 0
    check_heads(d)
    chained_any = False
    long_launch = False
    for t in range(3):
        items = d["groups"][t][1]          # TK_CR2: [gextra, follow, rows 0..2, players 0..2]
        marks = d["chains"][t]             # [chain, chained]
        assert len(items) == len(marks)
        leads = [i for i, it in enumerate(items) if it[1] == 0]
        for i, it in enumerate(items):
            if it[1] == 1:
                assert marks[i] == [0, 0], "followers carry no chain marks"
        g = 0
        blocks = 0
        while g < len(leads):
            head = leads[g]
            assert marks[head][1] == 0, "a chain starts with an unchained leader"
            c = marks[head][0]
            assert 0 <= c <= CHAIN_MAX - 1
            for m in leads[g + 1:g + 1 + c]:
                assert marks[m] == [0, 1]
                assert items[m][2] == items[head][2] and items[m][5:7] == items[head][5:7]
            chained_any = chained_any or c > 0
            blocks += 1
            g += 1 + c
        assert blocks >= min(len(leads), CHAIN_BLOCKS)
        if len(leads) < 2 * CHAIN_BLOCKS:
            assert blocks == len(leads), "a launch of fewer than two chain lengths' worth of groups is not chained"
        long_launch = long_launch or len(leads) >= 2 * CHAIN_BLOCKS
    assert chained_any == long_launch
    assert long_launch == ((raises, bets) in ((2, 3), (3, 2)))
