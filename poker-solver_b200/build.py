"""Build the street-solver shared libraries in-tree with nvcc for sm_100a.

  poker-solver_b200/lib/libstreet_solve.so       SS_MAX_HANDS = 200  (reference struct layout)
  poker-solver_b200/lib/libstreet_solve_wide.so  SS_MAX_HANDS = 1326 (every 2-card combo)

Both export the C ABIs of include/street_solve.h and include/flop_solve.h.  The engine objects are
compiled once and linked into both; only the ABI translation unit differs.
The CUDA runtime is linked statically, so each library is self-contained.
"""
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIBDIR = os.path.join(PKG, "lib")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I", INCLUDE, "-I", CSRC]
ENGINE = ["ss_tree.cpp", "ss_plan.cpp", "ss_kernels.cu", "ss_engine.cu", "ss_rank_kernels.cu", "ss_noalloc.cu", "ss_batch.cu",
          "ss_leaf_plan.cpp", "ss_leaf.cu", "ss_narrow.cu", "fs_tree.cpp", "fs_engine.cu", "fs_abi.cpp"]
HEADERS = ["ss_engine.h", "ss_kernels.h", "ss_rank.cuh", "ss_session.h", "ss_leaf.h", "ss_leaf.cuh", "fs_engine.h"]
VARIANTS = {"libstreet_solve.so": 200, "libstreet_solve_wide.so": 1326}


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _nvcc(args, verbose):
    cmd = ["nvcc"] + args
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build(verbose=False, force=False, ptxas_info=False):
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, h) for h in ("street_solve.h",
                                                                                          "flop_solve.h")]
    objs = []
    for src in ENGINE:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        if force or _newer(o, [s] + hdrs):
            extra = ["-Xptxas", "-v"] if (ptxas_info and src.endswith(".cu")) else []
            _nvcc(COMMON + ARCH + extra + ["-c", s, "-o", o], verbose)
        objs.append(o)
    built = []
    for lib, hands in VARIANTS.items():
        s = os.path.join(CSRC, "ss_abi.cpp")
        o = os.path.join(BUILD, f"ss_abi_{hands}.o")
        if force or _newer(o, [s] + hdrs):
            _nvcc(COMMON + ARCH + [f"-DSS_MAX_HANDS={hands}", "-c", s, "-o", o], verbose)
        out = os.path.join(LIBDIR, lib)
        if force or _newer(out, objs + [o]):
            _nvcc(ARCH + ["-shared", "-Xcompiler", "-fPIC", "-o", out] + objs + [o], verbose)
        built.append(out)
    return built


if __name__ == "__main__":
    for p in build(verbose="-v" in sys.argv, force="--force" in sys.argv,
                   ptxas_info="--ptxas" in sys.argv):
        print(p)
