"""Host check of the three-opponent closed forms (k_term_cr3 and
k_term_sd3, the block phases of poker-solver_b200/csrc/ss_cr3.cuh): the
phases compiled with g++ (tests/native/cr3_emul, sd3_emul) and run one after
another over 256 emulated threads, against brute-force enumeration of the
pairwise disjoint opponent tuples for every traverser hand (the reference's
rules, street_solve.cu:771-823 folds, :936-1002 showdowns):
* folds / leaves: the FP64 mass to 1e-12 relative, the integer tuple count
  exactly, and exact zeros for hands without a tuple of positive products --
  on full-size decks (turn 48, river 47, flop 49 cards), with zeroed
  weights, a range the board touches, an opponent without positive reach,
  and tiny decks where most hands have no disjoint tuple;
* four-way showdowns: every class mass (win, 2-, 3-, 4-way ties, per pair of
  the first two opponents' weaker / tying parts and the third opponent's
  class) and the value, with ties from few rank levels up to every hand
  tying, a pot / 3 equal to the bet, and a bet of 0; counts exact and the
  classes without a tuple exactly 0;
* sparse four-way showdowns (tests/native/sd3inc_emul): the weaker parts'
  tables grown hand by hand along the rank levels equal a direct build at
  every level (FP64 fields to 1e-13 relative, masks and counts exactly), and
  the pairs with a tying part evaluated from those tables and the tying
  hands' lists equal each pair's own tables' class masses, with exact tuple
  counts and classes without a tuple exactly 0;
* both kernels' blocks driven by the planner's own work items and tables
  for seeded 4-player rivers and a 4-player turn (tests/native/term3_emul,
  with ss_plan.cpp and ss_tree.cpp): hand codes, pair tables, rank
  positions, tie-group walk and term groups, every traverser hand against
  enumeration with the planner's strengths, to 1e-12."""
import json
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HERE = os.path.dirname(os.path.abspath(__file__))


def _build(tmp_path_factory, name):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    out = str(tmp_path_factory.mktemp("cr3") / name)
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-I", os.path.join(ROOT, "include"),
                    "-I", os.path.join(ROOT, "poker-solver_b200", "csrc"),
                    os.path.join(HERE, "native", name + ".cpp"), "-o", out], check=True)
    return out


@pytest.fixture(scope="module")
def emul(tmp_path_factory):
    return _build(tmp_path_factory, "cr3_emul")


@pytest.fixture(scope="module")
def sd3(tmp_path_factory):
    return _build(tmp_path_factory, "sd3_emul")


@pytest.mark.parametrize("args", [
    (1, 47, 20, 0.3, 6, 100, 25),     # river deck, some ties
    (2, 48, 24, 0.0, 3, 150, 50),     # few rank levels: many ties
    (3, 10, 30, 0.2, 2, 75, 25),      # pot / 3 equals the bet: 3-way ties pay exactly 0
    (4, 8, 20, 0.0, 1, 90, 30),       # every hand ties
    (5, 47, 18, 0.5, 40, 300, 0),     # a bet of 0: losses pay exactly 0
])
def test_four_way_showdown_classes_against_enumeration(sd3, args):
    r = subprocess.run([sd3] + [str(a) for a in args], check=True, capture_output=True, text=True)
    d = json.loads(r.stdout)
    assert d["zero_bad"] == 0
    assert d["max_rel_err"] <= 1e-12
    assert d["hands"] > 0 and d["empty_classes"] > 0


@pytest.mark.parametrize("args,min_zero", [
    ((1, 47, 24, 0.3), 0),        # river deck
    ((2, 48, 30, 0.6), 0),        # turn deck, most weights zero
    ((3, 49, 20, 0.0), 0),        # flop deck
    ((6, 47, 30, 0.2, 1), 30),    # the second opponent has no positive reach: every mass is 0
    ((8, 7, 21, 0.0), 10),        # 7 cards: only hands holding a board card leave room for three opponents
    ((9, 8, 28, 0.0), 0),
    ((12, 10, 45, 0.7), 0),
])
def test_closed_form_against_enumeration(emul, args, min_zero):
    r = subprocess.run([emul] + [str(a) for a in args], check=True, capture_output=True, text=True)
    d = json.loads(r.stdout)
    assert d["count_mismatches"] == 0
    assert d["max_rel_err"] <= 1e-12
    assert d["zero_bad"] == 0
    assert d["zero_hands"] >= min_zero


@pytest.fixture(scope="module")
def term3(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    out = str(tmp_path_factory.mktemp("cr3") / "term3_emul")
    csrc = os.path.join(ROOT, "poker-solver_b200", "csrc")
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-I", os.path.join(ROOT, "include"), "-I", csrc,
                    os.path.join(HERE, "native", "term3_emul.cpp"), os.path.join(csrc, "ss_plan.cpp"),
                    os.path.join(csrc, "ss_tree.cpp"), "-o", out], check=True)
    return out


@pytest.mark.parametrize("args", [
    (1, 5, 20, 0.2, 20),     # 4-player river: three-opponent folds and four-way showdowns
    (2, 5, 24, 0.0, 20),
    (4, 5, 30, 0.5, 10),     # half the reach rows' entries zero
    (3, 4, 18, 0.3, 12),     # 4-player turn: folds and grouped continuation leaves
])
def test_kernel_blocks_on_planned_items(term3, args):
    r = subprocess.run([term3] + [str(a) for a in args], check=True, capture_output=True, text=True)
    d = json.loads(r.stdout)
    assert d["items"] > 0 and d["hands"] > 0
    assert d["max_rel_err"] <= 1e-12
    assert d["zero_bad"] == 0


@pytest.fixture(scope="module")
def sd3inc(tmp_path_factory):
    return _build(tmp_path_factory, "sd3inc_emul")


@pytest.mark.parametrize("args", [
    (1, 20, 60, 0.3, 6),       # small deck, several hands per level
    (2, 47, 120, 0.5, 12),     # river deck, half the weights zero
    (3, 12, 40, 0.0, 3),       # few levels: large tying parts
    (4, 30, 200, 0.6, 30),     # many levels, sparse
])
def test_sparse_showdown_steps_against_direct_builds(sd3inc, args):
    r = subprocess.run([sd3inc] + [str(a) for a in args], check=True, capture_output=True, text=True)
    d = json.loads(r.stdout)
    assert d["hands"] > 0
    assert d["bad"] == 0
    assert d["max_table_err"] <= 1e-13
    assert d["max_rel_err"] <= 1e-12
