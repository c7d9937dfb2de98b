"""Golden vectors of the reference's range update (python/range_narrowing.py,
RangeNarrower.update / remove_folded_hands / get_hand_count), made by
importing the reference module itself.  Run where the reference checkout is
present:

    python tests/golden/make_narrow_golden.py [REFERENCE_ROOT]

Writes tests/golden/narrow_cases.json.gz: seeded starting ranges (with zero
weights, entries stored with c0 > c1 and combos missing from the
probabilities) and sequences of updates with their probability dictionaries,
and after every step the reference's weights (as float.hex strings, so the
comparison is bit for bit), hand count and action log.
"""
import gzip
import importlib.util
import json
import os
import random
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def _ref_root():
    if len(sys.argv) > 1:
        return sys.argv[1]
    spec = importlib.util.spec_from_file_location("oracle_build_ref", os.path.join(ROOT, "oracle", "build_ref.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.REF


def load_reference():
    path = os.path.join(_ref_root(), "python", "range_narrowing.py")
    spec = importlib.util.spec_from_file_location("ref_range_narrowing", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def make_case(rng, ref, uniform):
    nr = ref.RangeNarrower()
    if uniform:
        nr.set_uniform_range("villain")
    else:
        hands = []
        for a in range(52):
            for b in range(a + 1, 52):
                if rng.random() < 0.3:
                    w = 0.0 if rng.random() < 0.15 else rng.random()
                    hands.append((b, a, w) if rng.random() < 0.05 else (a, b, w))
        nr.set_initial_range("villain", hands)
    start = [[c0, c1, float(w).hex()] for c0, c1, w in nr._ranges["villain"]]
    steps = []
    for k in range(3):
        probs = {}
        levels = [0.0, 0.25, 0.5, 1.0] if k == 0 else None
        for c0, c1, _ in nr._ranges["villain"]:
            key = (min(c0, c1), max(c0, c1))
            if rng.random() < 0.9:
                probs[key] = rng.choice(levels) if levels else round(rng.random(), 3) * (rng.random() < 0.8)
        action = ["Check", "Bet 75%", "Call"][k]
        nr.update("villain", action, probs)
        steps.append({"action": action,
                      "probs": [[a, b, float(p).hex()] for (a, b), p in sorted(probs.items())],
                      "weights": [float(w).hex() for _, _, w in nr._ranges["villain"]],
                      "hand_count": nr.get_hand_count("villain"),
                      "log": list(nr.get_action_log("villain"))})
    fold = {(min(c0, c1), max(c0, c1)): rng.random() for c0, c1, _ in nr._ranges["villain"]}
    nr.remove_folded_hands("villain", fold)
    return {"uniform": uniform, "start": start, "steps": steps,
            "fold_probs": [[a, b, float(p).hex()] for (a, b), p in sorted(fold.items())],
            "after_fold": [[c0, c1, float(w).hex()] for c0, c1, w in nr._ranges["villain"]]}


def main():
    ref = load_reference()
    rng = random.Random(20260)
    cases = [make_case(rng, ref, uniform) for uniform in (True, False, False)]
    out = os.path.join(HERE, "narrow_cases.json.gz")
    with gzip.open(out, "wt") as f:
        json.dump(cases, f, separators=(",", ":"))
    print(out, os.path.getsize(out))


if __name__ == "__main__":
    main()
