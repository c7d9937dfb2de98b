"""Build the oracle's C restatement into oracle/lib/liboracle.so.

TEST INFRASTRUCTURE ONLY: the library is the checker used by tests/, the smoke
check and bench.py's CPU baseline; the product never loads it.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "lib", "liboracle.so")
SRCS = ["ss_oracle.c", "ss_oracle_impl.h", "ss_oracle.h", "oracle_eval.h", "oracle_bench.c", "fs_oracle.c",
        "fs_oracle_impl.h"]


def build(force=False):
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    srcs = [os.path.join(HERE, s) for s in SRCS if os.path.exists(os.path.join(HERE, s))]
    if not force and os.path.exists(LIB) and all(
            os.path.getmtime(s) <= os.path.getmtime(LIB) for s in srcs):
        return LIB
    c_srcs = [s for s in srcs if s.endswith(".c")]
    subprocess.run(["gcc", "-O2", "-fPIC", "-shared", "-fopenmp", "-Wall", "-o", LIB] + c_srcs
                   + ["-lm"], check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
