"""Host check of the three-counted-opponent closed form (k_term_cr3, the
block phases of poker-solver_b200/csrc/ss_cr3.cuh): the phases compiled
with g++ into tests/native/cr3_emul and run one after another over 256
emulated threads, against brute-force enumeration of the pairwise disjoint
opponent tuples for every traverser hand (the reference's rule,
street_solve.cu:771-823): the FP64 mass to 1e-12 relative, the integer
tuple count exactly, and exact zeros for hands without a tuple of positive
products -- on full-size decks (turn 48, river 47, flop 49 cards), with
zeroed weights, a range the board touches, an opponent without positive
reach, and tiny decks where most hands have no disjoint tuple."""
import json
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def emul(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    out = str(tmp_path_factory.mktemp("cr3") / "cr3_emul")
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-I", os.path.join(ROOT, "include"),
                    "-I", os.path.join(ROOT, "poker-solver_b200", "csrc"),
                    os.path.join(HERE, "native", "cr3_emul.cpp"), "-o", out], check=True)
    return out


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
