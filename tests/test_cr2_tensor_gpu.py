"""The tensor-core (tcgen05) form of the two-opponent terminals, taken with
SSB_CR2_TENSOR=1 (read once per process, so the cases run in a child
process): the strict and envelope 3-player turn cases of test_parity_gpu
against the oracle, and the strict cases' average strategies through the
default (mma.sync) form within the parity tolerance."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))

CHILD = r"""
import json, sys
sys.path[:0] = {paths!r}
import numpy as np
import test_parity_gpu as tp
import workloads as wl
from oracle.oracle import Oracle
oracle = Oracle()
out = {{}}
for name, seed, nh, iters, over, mode in [("turn3", 3, 12, 10, tp.SMALL_TURN, "strict"),
                                           ("turn3", 4, 10, 3, {{}}, "strict"),
                                           ("turn3", 3, 24, 12, {{}}, "envelope")]:
    cfg = wl.config(name, seed=seed, num_hands=nh, **over)
    ours, lv = tp.solve(cfg, iters)
    r32, r64 = tp.oracle_pair(oracle, cfg, iters, lv)
    if mode == "strict":
        tp.strict(ours, r32)
    else:
        tp.envelope(ours, r32, r64)
    out[f"{{name}}-{{seed}}-{{nh}}"] = ours["avg_strategies"].ravel().tolist()[:4000]
print("RESULT " + json.dumps(out))
"""


def run_child(tensor):
    from conftest import PKG, ROOT
    env = dict(os.environ)
    env["SSB_CR2_TENSOR"] = "1" if tensor else "0"
    code = CHILD.format(paths=[ROOT, PKG, HERE])
    p = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=900)
    assert p.returncode == 0, p.stdout[-3000:] + p.stderr[-3000:]
    line = [l for l in p.stdout.splitlines() if l.startswith("RESULT ")][-1]
    return json.loads(line[7:])


@pytest.mark.gpu
def test_tensor_form_parity_and_agreement():
    tc = run_child(True)
    mm = run_child(False)
    for k in tc:
        if k.endswith("-24"):
            continue   # the envelope case: rounding-order differences grow past 1e-4 by design
        d = np.abs(np.array(tc[k]) - np.array(mm[k])).max()
        assert d <= 1e-4, f"{k}: tensor vs mma.sync forms differ by {d}"
