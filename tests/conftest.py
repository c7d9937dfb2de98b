"""Test configuration: the `gpu` marker and import paths.

GPU tests call the CUDA path through the C ABI and compare with the oracle;
everything else runs on CPU.  The oracle is imported only here in tests/ as
the checker."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "poker-solver_b200")
for p in (ROOT, PKG, os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the sm_100a kernels")


def _have_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


HAVE_GPU = _have_gpu()


# Files run after all others, in this order: the continuation-value
# producer's and the three-opponent closed form's GPU tests after the rest
# of the solver's (so that under -x a failure there cannot keep the solver's
# tests from running), the no-allocation entry point last.  The sort is
# stable: everything else keeps file order.
_RUN_LATE = {"test_leaf_values_gpu.py": 1, "test_cr3_gpu.py": 2, "test_zz_no_alloc.py": 3}


def pytest_collection_modifyitems(config, items):
    items.sort(key=lambda it: _RUN_LATE.get(os.path.basename(str(it.fspath)), 0))
    if HAVE_GPU:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session", autouse=True)
def built_libraries():
    """Build the product libraries and the oracle once if they are missing
    (the GPU box receives them prebuilt)."""
    import importlib.util
    lib = os.path.join(PKG, "lib", "libstreet_solve.so")
    if not os.path.exists(lib) or not os.path.exists(os.path.join(PKG, "lib", "libstreet_solve_wide.so")):
        spec = importlib.util.spec_from_file_location("ssb_build", os.path.join(PKG, "build.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        mod.build()
    yield
