"""Build the reference's own code for the hot path into oracle/_ref/.

TEST INFRASTRUCTURE ONLY.  Compiles, from the reference sources where they lie
(default /root/reference, override with REF_ROOT), without running the
reference's build system:

  libref_handeval.so          src/hand_eval.h behind oracle/ref_handeval.c
  libref_solver.so            src/solver.c (2-player CPU Linear CFR), -O2 -fopenmp
  ref_h{H}_r{R}/libref_street_solve_cpu.so
                              src/cuda/street_solve.cu run on the CPU: the kernel
                              launches <<<g, b>>> are rewritten into host loops
                              (SHIM_LAUNCH, oracle/ref_shim/cuda_runtime.h) and the
                              header limits SS_MAX_HANDS / SS_MAX_RAISES are set to
                              H / R in a generated copy of street_solve.cuh.
  libref_street_solve_gpu.so  src/cuda/street_solve.cu unmodified, nvcc sm_100a
                              (stock limits: 200 hands, 3 raises); for parity runs
                              on a B200 at <= 200 hands.
  libref_flop_solve_gpu.so    src/cuda/flop_solve.cu unmodified, nvcc sm_100a: its
                              tree builder (host code) pins fs_build_tree here,
                              its solve pins fs_solve_gpu on a B200.
  wrapper/python/             python/street_solver_gpu.py and python/solver.py,
                              copied unmodified: the reference's own ctypes
                              consumer of the C ABI, which the drop-in test runs
                              against this repository's library.

Everything generated lands under oracle/_ref/, which git ignores.
"""
import os
import re
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
# the reference checkout: REF_ROOT, else where this build keeps it (the only
# place any script of the repository names that location)
REF = os.environ.get("REF_ROOT", "/root/reference")

# (SS_MAX_HANDS, SS_MAX_RAISES) variants of the CPU-shim build
VARIANTS = [(200, 3), (200, 2), (1326, 2), (1326, 3)]


def _run(cmd):
    subprocess.run(cmd, check=True)


def _fresh(target, sources):
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(s) <= t for s in sources)


def build_handeval():
    out = os.path.join(OUT, "libref_handeval.so")
    src = os.path.join(HERE, "ref_handeval.c")
    hdr = os.path.join(REF, "src", "hand_eval.h")
    if _fresh(out, [src, hdr]):
        return out
    _run(["gcc", "-O2", "-fopenmp", "-fPIC", "-shared", "-I", os.path.join(REF, "src"), src, "-o", out])
    return out


def build_solver():
    out = os.path.join(OUT, "libref_solver.so")
    src = os.path.join(REF, "src", "solver.c")
    if _fresh(out, [src]):
        return out
    _run(["gcc", "-O2", "-fopenmp", "-fPIC", "-shared", "-I", os.path.join(REF, "src"),
          src, "-o", out, "-lm"])
    return out


_LAUNCH = re.compile(r"(\w+)\s*<<<\s*([^,]+?)\s*,\s*(.+?)\s*>>>\s*\(")


def build_shim(max_hands, max_raises):
    vdir = os.path.join(OUT, f"ref_h{max_hands}_r{max_raises}")
    os.makedirs(vdir, exist_ok=True)
    out = os.path.join(vdir, "libref_street_solve_cpu.so")
    cu = os.path.join(REF, "src", "cuda", "street_solve.cu")
    cuh = os.path.join(REF, "src", "cuda", "street_solve.cuh")
    shim = os.path.join(HERE, "ref_shim", "cuda_runtime.h")
    if _fresh(out, [cu, cuh, shim, __file__]):
        return out
    hdr = open(cuh).read()
    hdr = re.sub(r"#define SS_MAX_HANDS\s+\d+", f"#define SS_MAX_HANDS      {max_hands}", hdr)
    hdr = re.sub(r"#define SS_MAX_RAISES\s+\d+", f"#define SS_MAX_RAISES     {max_raises}", hdr)
    open(os.path.join(vdir, "street_solve.cuh"), "w").write(hdr)
    body = open(cu).read()
    body, n = _LAUNCH.subn(r"SHIM_LAUNCH(\1, \2, \3, ", body)
    if n < 8:
        raise RuntimeError(f"expected >= 8 kernel launches in street_solve.cu, rewrote {n}")
    gen = os.path.join(vdir, "street_solve_shim.cpp")
    with open(gen, "w") as f:
        f.write("#include <cuda_runtime.h>\n")
        f.write("thread_local shim_dim3 threadIdx, blockIdx;\n")
        f.write(body)
    _run(["g++", "-O2", "-fPIC", "-shared", "-w", "-I", os.path.join(HERE, "ref_shim"),
          gen, "-o", out])
    return out


def build_gpu():
    out = os.path.join(OUT, "libref_street_solve_gpu.so")
    cu = os.path.join(REF, "src", "cuda", "street_solve.cu")
    if _fresh(out, [cu]):
        return out
    if shutil.which("nvcc") is None:
        return None
    _run(["nvcc", "-O2", "-gencode", "arch=compute_100a,code=sm_100a", "-shared",
          "-Xcompiler", "-fPIC", "-w", cu, "-o", out])
    return out


def build_flop_gpu():
    out = os.path.join(OUT, "libref_flop_solve_gpu.so")
    cu = os.path.join(REF, "src", "cuda", "flop_solve.cu")
    if _fresh(out, [cu]):
        return out
    if shutil.which("nvcc") is None:
        return None
    _run(["nvcc", "-O2", "-gencode", "arch=compute_100a,code=sm_100a", "-shared",
          "-Xcompiler", "-fPIC", "-w", cu, "-o", out])
    return out


def build_wrapper():
    """The reference's Python consumer of the C ABI, unmodified (it imports
    card helpers from solver.py and loads <root>/build/street_solve.so)."""
    out = os.path.join(OUT, "wrapper", "python")
    os.makedirs(out, exist_ok=True)
    for name in ("street_solver_gpu.py", "solver.py"):
        src = os.path.join(REF, "python", name)
        dst = os.path.join(out, name)
        if not _fresh(dst, [src]):
            shutil.copyfile(src, dst)
    return out


def main():
    if not os.path.isdir(os.path.join(REF, "src", "cuda")):
        print(f"reference sources not found under {REF}; nothing to build", file=sys.stderr)
        return 0
    os.makedirs(OUT, exist_ok=True)
    built = [build_handeval(), build_solver()]
    for h, r in VARIANTS:
        built.append(build_shim(h, r))
    built.append(build_gpu())
    built.append(build_flop_gpu())
    built.append(build_wrapper())
    for b in built:
        if b:
            print(os.path.relpath(b, HERE))
    return 0


if __name__ == "__main__":
    sys.exit(main())
