"""The ragged batch's overlap check on column output ranges (batch_layout.h, used by
oco_batch_create / oco_batch_bind), compiled for the host and compared with a brute-force
pairwise check."""
import ctypes
import itertools
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BUILD = os.path.join(ROOT, "tests", "_build")
I64P = ctypes.POINTER(ctypes.c_int64)


@pytest.fixture(scope="module")
def lib():
    os.makedirs(BUILD, exist_ok=True)
    out = os.path.join(BUILD, "libbatch_layout_host.so")
    cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-I", os.path.join(ROOT, "ocotillo_b200", "csrc"),
           "-o", out, os.path.join(ROOT, "tests", "batch_layout_host.cpp")]
    subprocess.run(cmd, check=True, capture_output=True)
    h = ctypes.CDLL(out)
    h.batch_first_overlap.argtypes = [I64P, I64P, ctypes.c_int64, I64P]
    return h


def first_overlap(h, off, length):
    off = np.ascontiguousarray(off, dtype=np.int64)
    length = np.ascontiguousarray(length, dtype=np.int64)
    pair = np.zeros(2, dtype=np.int64)
    h.batch_first_overlap(off.ctypes.data_as(I64P), length.ctypes.data_as(I64P), len(off), pair.ctypes.data_as(I64P))
    return int(pair[0]), int(pair[1])


def meet(off, length, i, j):
    return length[i] > 0 and length[j] > 0 and off[i] < off[j] + length[j] and off[j] < off[i] + length[i]


def test_dense_packing_has_no_overlap(lib):
    from ocotillo_b200 import dense_batch_offsets
    nz, nw = [2, 512, 37, 1024, 64], [1, 256, 3, 17, 1024]
    o = dense_batch_offsets(nz, nw)
    assert first_overlap(lib, o["u_off"], [(a + 6) * b for a, b in zip(nz, nw)]) == (-1, -1)
    assert first_overlap(lib, o["kv_off"], [a * b for a, b in zip(nz, nw)]) == (-1, -1)
    assert first_overlap(lib, o["flux_off"], nw) == (-1, -1)


def test_known_cases(lib):
    assert first_overlap(lib, [0], [5]) == (-1, -1)
    assert first_overlap(lib, [0, 5], [5, 5]) == (-1, -1)        # touching ends
    assert first_overlap(lib, [0, 4], [5, 5]) == (0, 1)
    assert first_overlap(lib, [7, 7], [1, 1]) == (0, 1)          # same start
    assert first_overlap(lib, [10, 0, 3], [2, 100, 1]) in {(0, 1), (1, 2)}  # one range covers two
    assert first_overlap(lib, [0, 2, 0], [2, 2, 0]) == (-1, -1)  # empty range meets nothing
    assert first_overlap(lib, [2**56, 2**56 - 1], [2**62, 2]) == (0, 1)


def test_random_layouts_against_pairwise(lib):
    rng = np.random.default_rng(5)
    for trial in range(400):
        n = int(rng.integers(1, 12))
        length = rng.integers(0, 6, n)
        off = rng.integers(0, 30, n) if trial % 2 else np.concatenate([[0], np.cumsum(length)[:-1]])
        if trial % 5 == 0 and n > 1:  # dense packing with one column moved into its neighbour
            k = int(rng.integers(1, n))
            off = off.copy()
            off[k] -= int(rng.integers(0, 3))
        got = first_overlap(lib, off, length)
        pairs = [(i, j) for i, j in itertools.combinations(range(n), 2) if meet(off, length, i, j)]
        if pairs:
            assert got[0] < got[1] and meet(off, length, *got), (off, length, got)
        else:
            assert got == (-1, -1), (off, length, got)
