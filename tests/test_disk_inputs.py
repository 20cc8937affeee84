"""The synthetic disk generator (disk_core.h; oco_disk_inputs on the host, oco_disk_inputs_device
on the GPU): the reference's disk model (source/disk.f90:42-129) and a seeded lognormal density
perturbation from Philox4x32-10.  CPU checks: the generator's known-answer vectors, the normal
deviates' moments, agreement with the deck reader's synthetic disk (which uses the C library's
exp), and argument checks."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BUILD = os.path.join(ROOT, "tests", "_build")


@pytest.fixture(scope="module")
def host():
    os.makedirs(BUILD, exist_ok=True)
    out = os.path.join(BUILD, "libphilox_host.so")
    subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off", "-I",
                    os.path.join(ROOT, "ocotillo_b200", "csrc"), "-o", out, os.path.join(ROOT, "tests", "philox_host.cpp")],
                   check=True, capture_output=True)
    h = ctypes.CDLL(out)
    U = ctypes.POINTER(ctypes.c_uint32)
    h.philox_host.argtypes = [U, ctypes.c_uint32, ctypes.c_uint32, U]
    h.normals_host.argtypes = [ctypes.c_uint64, ctypes.c_int64, ctypes.POINTER(ctypes.c_double)]
    return h


# Known-answer vectors of Philox4x32-10 published with the generator (Random123's kat_vectors):
# (counter, key) -> output.
KAT = [((0, 0, 0, 0), (0, 0), (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
       ((0xffffffff,) * 4, (0xffffffff, 0xffffffff), (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
       ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
        (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1))]


@pytest.mark.parametrize("ctr,key,want", KAT)
def test_philox_known_answers(host, ctr, key, want):
    c = (ctypes.c_uint32 * 4)(*ctr)
    o = (ctypes.c_uint32 * 4)()
    host.philox_host(c, key[0], key[1], o)
    assert tuple(o) == want


def test_normal_deviates(host):
    n = 1 << 20
    x = np.empty(n)
    host.normals_host(12345, n, x.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    assert abs(x.mean()) < 5e-3 and abs(x.std() - 1.0) < 5e-3
    assert abs((np.abs(x) < 1.0).mean() - 0.6827) < 3e-3  # one-sigma mass
    y = np.empty(n)
    host.normals_host(12346, n, y.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    assert abs(np.corrcoef(x, y)[0, 1]) < 5e-3


def test_disk_without_perturbation_is_the_reference_disk():
    """sigma_dex = 0 gives the deck reader's synthetic disk (NongreyAGN deck), to the last ulp
    or two: the deck reader calls the C library's exp, this generator the correctly rounded one."""
    from conftest import SAMPLES
    from ocotillo_b200 import deck_block_inputs, disk_inputs
    d = deck_block_inputs(os.path.join(SAMPLES, "NongreyAGN"))
    rho_d, T_d = d["rho"], d["T"]
    import re
    text = open(os.path.join(SAMPLES, "NongreyAGN", "input.in")).read()
    vals = dict((k, float(v.replace("d", "e").replace("D", "e"))) for k, v in
                re.findall(r"(\w+)\s*=\s*([-+0-9.eEdD]+)", text))
    kw = {k: vals[k] for k in ("z0", "z1", "rho0", "H", "rho_floor", "midTemp", "sigma", "floorTemp", "isoTemp")
          if k in vals}
    rho, T, dz = disk_inputs(rho_d.shape, **kw)
    assert dz == d["dz"]
    assert np.abs(rho / rho_d - 1).max() <= 4.5e-16
    assert np.abs(T / T_d - 1).max() <= 4.5e-16


def test_perturbation_is_lognormal_and_seeded():
    from ocotillo_b200 import disk_inputs
    shape = (8, 8, 512)
    r0, T0, _ = disk_inputs(shape)
    r1, T1, _ = disk_inputs(shape, sigma_dex=0.3, seed=3)
    r2, _, _ = disk_inputs(shape, sigma_dex=0.3, seed=3)
    r3, _, _ = disk_inputs(shape, sigma_dex=0.3, seed=4)
    assert np.array_equal(T0, T1) and np.array_equal(r1, r2) and not np.array_equal(r1, r3)
    d = np.log10(r1 / r0)
    assert abs(d.mean()) < 0.01 and abs(d.std() - 0.3) < 0.01


def test_bad_parameters_refused():
    from ocotillo_b200 import OcoError, disk_inputs
    with pytest.raises(OcoError):
        disk_inputs((1, 1, 1))
    with pytest.raises(OcoError):
        disk_inputs((1, 1, 8), H=0.0)
    with pytest.raises(ValueError):
        disk_inputs((1, 1, 8), Hh=1.0)
