"""The device 7-card ranker against the reference evaluator src/hand_eval.h:
all 133,784,560 sets through the order-independent checksum recorded from
the reference (tests/golden/hand_rank_all.json), and a random sample value
for value."""
import ctypes
import json
import os

import numpy as np
import pytest

import street_solver_gpu as ssg

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.gpu
def test_device_ranker_all_hands():
    lib = ssg.load_library(200)
    ref = json.load(open(os.path.join(GOLDEN, "hand_rank_all.json")))
    chk = ctypes.c_ulonglong()
    hist = (ctypes.c_ulonglong * 10)()
    assert lib.ss_rank7_checksum(ctypes.byref(chk), hist) == 0, ssg.last_error(lib)
    assert list(hist) == ref["category_counts"]
    assert f"{chk.value:#018x}" == ref["checksum"]


@pytest.mark.gpu
def test_device_ranker_sample():
    lib = ssg.load_library(200)
    g = np.load(os.path.join(GOLDEN, "hand_rank_sample.npz"))
    cards = np.ascontiguousarray(g["cards"], np.int32)
    out = np.zeros(len(cards), np.uint32)
    rc = lib.ss_rank7_batch(cards.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), len(cards),
                            out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint)))
    assert rc == 0, ssg.last_error(lib)
    assert np.array_equal(out, g["strength"])


def test_ranker_rejects_bad_cards():
    lib = ssg.load_library(200)
    cards = np.full((1, 7), 99, np.int32)
    out = np.zeros(1, np.uint32)
    rc = lib.ss_rank7_batch(cards.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), 1,
                            out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint)))
    assert rc == -1
