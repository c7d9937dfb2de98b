"""The host side of range narrowing against the reference module's own
outputs (tests/golden/narrow_cases.json.gz, made by make_narrow_golden.py
from python/range_narrowing.py): every weight bit for bit after each update,
the hand counts, the action log and the fold filter."""
import gzip
import json
import os

import pytest

import range_narrowing as rn

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "narrow_cases.json.gz")


def cases():
    with gzip.open(GOLDEN, "rt") as f:
        return json.load(f)


@pytest.mark.parametrize("case", cases(), ids=lambda c: "uniform" if c["uniform"] else "initial")
def test_updates_match_reference(case):
    nr = rn.RangeNarrower()
    if case["uniform"]:
        nr.set_uniform_range("villain")
    else:
        nr.set_initial_range("villain", [(a, b, float.fromhex(w)) for a, b, w in case["start"]])
    assert [[a, b, float(w).hex()] for a, b, w in nr._ranges["villain"]] == case["start"]
    for st in case["steps"]:
        probs = {(a, b): float.fromhex(p) for a, b, p in st["probs"]}
        nr.update("villain", st["action"], probs)
        assert [float(w).hex() for _, _, w in nr._ranges["villain"]] == st["weights"]
        assert nr.get_hand_count("villain") == st["hand_count"]
        assert nr.get_action_log("villain") == st["log"]
    nr.remove_folded_hands("villain", {(a, b): float.fromhex(p) for a, b, p in case["fold_probs"]})
    assert [[a, b, float(w).hex()] for a, b, w in nr._ranges["villain"]] == case["after_fold"]


def test_helpers():
    hands = rn.generate_all_hands([0, 1, 2])
    assert len(hands) == 49 * 48 // 2 and all(a < b and w == 1.0 for a, b, w in hands)
    probs = rn.make_blueprint_probs({"AhKs": {"actions": [{"action": "Check", "frequency": 0.25},
                                                          {"action": "Bet 75%", "frequency": 0.75}]}}, "bet")
    assert list(probs.values()) == [0.75]
    nr = rn.RangeNarrower()
    nr.update("nobody", "Check", {})      # unknown player: no-op, as in the reference
    assert nr.get_weighted_hands("nobody") == []
