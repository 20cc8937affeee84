"""The deck layer (input construction, Ew.d editing, Fortran records) on the CPU, against the
oracle's restatement of the reference's driver: the same bytes for every deck's root-block
inputs, the same text for every formatted value; and its refusals of bad decks as error codes."""
import os
import shutil

import numpy as np
import pytest

from conftest import DECKS, SAMPLES


@pytest.mark.parametrize("deck", DECKS)
def test_block_inputs_match_oracle(oracle, tmp_path, deck):
    from ocotillo_b200 import deck_block_inputs
    rc, msg = oracle.run_deck(os.path.join(SAMPLES, deck), str(tmp_path), backend="glibc")
    assert rc == 0, msg
    meta = open(tmp_path / "inputs_meta.txt").read().split()
    nx, ny, nz, nw = (int(v) for v in meta[:4])
    d = deck_block_inputs(os.path.join(SAMPLES, deck))
    assert (d["nxloc"], d["nyloc"], d["nz"], d["nw"]) == (nx, ny, nz, nw)
    assert d["dz"] == float(meta[4]) and d["lgrey"] == int(meta[5])
    assert d["sigma_grey"] == float(meta[6]) and d["fully_ionized_T"] == float(meta[7])
    assert np.array_equal(d["rho"].ravel(), np.fromfile(tmp_path / "inputs_rho.bin"))
    assert np.array_equal(d["T"].ravel(), np.fromfile(tmp_path / "inputs_T.bin"))
    assert np.array_equal(d["wa"], np.fromfile(tmp_path / "inputs_wa.bin"))


def test_format_e_matches_oracle(oracle):
    from ocotillo_b200 import format_e
    rng = np.random.default_rng(3)
    vals = list(10.0 ** rng.uniform(-320, 308, 4000) * rng.choice([-1, 1], 4000))
    vals += [0.0, -0.0, 1.0, 9.99995, 9.999949999, 0.1, 1e-100, 9.99999e99, 1e100, 5e-324, 1.7976931348623157e308,
             float("inf"), float("-inf"), float("nan"), 123456.5, 0.000123455]
    for v in vals:
        assert format_e(v) == oracle.format_e(v), v
    assert format_e(1.5e-101) == "    0.15000-100" and format_e(1.5e-100) == "    0.15000E-99"


def test_deck_errors(tmp_path):
    from ocotillo_b200 import OcoError, deck_block_inputs
    with pytest.raises(OcoError) as e:
        deck_block_inputs(str(tmp_path))
    assert e.value.code == -9  # EIO: no resolution.in
    d = tmp_path / "grey"
    shutil.copytree(os.path.join(SAMPLES, "GreyIsothermal"), d)
    txt = open(d / "resolution.in").read().replace("nw=1", "nw=3")
    open(d / "resolution.in", "w").write(txt)
    with pytest.raises(OcoError) as e:
        deck_block_inputs(str(d))
    assert e.value.code == -4  # EGREY, flux_feautrier.f90:84-87
    a = tmp_path / "athena"
    shutil.copytree(os.path.join(SAMPLES, "ReadFromAthena"), a)
    with pytest.raises(OcoError) as e:
        deck_block_inputs(str(a), snapshot="0001")
    assert e.value.code == -9  # missing snapshot file, read_athena.f90:112-116


def test_fortran_records_roundtrip(tmp_path):
    """The record reader against hand-made gfortran records, including a split record."""
    from ocotillo_b200 import read_fortran_records
    p = tmp_path / "r.bin"
    a = np.arange(5, dtype=np.float64).tobytes()
    b = b"x" * 7
    with open(p, "wb") as f:
        n = len(a).to_bytes(4, "little", signed=True)
        f.write(n + a + n)
        # one record of 7 bytes split as 3 + 4: leading markers -3, 4; trailing 3, -4
        f.write((-3).to_bytes(4, "little", signed=True) + b[:3] + (3).to_bytes(4, "little", signed=True))
        f.write((4).to_bytes(4, "little", signed=True) + b[3:] + (-4).to_bytes(4, "little", signed=True))
    recs = read_fortran_records(str(p))
    assert recs == [a, b]


@pytest.fixture(scope="module")
def record_writer():
    import ctypes
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    build = os.path.join(root, "tests", "_build")
    os.makedirs(build, exist_ok=True)
    out = os.path.join(build, "libfortran_records_host.so")
    subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-I", os.path.join(root, "ocotillo_b200", "csrc"),
                    "-o", out, os.path.join(root, "tests", "fortran_records_host.cpp")], check=True, capture_output=True)
    h = ctypes.CDLL(out)
    h.append_fortran_record.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_size_t, ctypes.c_size_t]
    return h


def test_fortran_record_writer_splits_into_subrecords(record_writer, tmp_path):
    """The writer the deck uses for its binary outputs, with a small subrecord limit standing in
    for gfortran's 2147483639 bytes: exact markers of a split record, and every size and limit
    read back by the reader."""
    from ocotillo_b200 import read_fortran_records
    le = lambda v: int(v).to_bytes(4, "little", signed=True)
    p = tmp_path / "split.bin"
    assert record_writer.append_fortran_record(str(p).encode(), b"abcdefg", 7, 3) == 0
    assert p.read_bytes() == (le(-3) + b"abc" + le(3) + le(-3) + b"def" + le(-3) + le(1) + b"g" + le(-1))
    q = tmp_path / "whole.bin"
    assert record_writer.append_fortran_record(str(q).encode(), b"abcdefg", 7, 2147483639) == 0
    assert q.read_bytes() == le(7) + b"abcdefg" + le(7)
    rng = np.random.default_rng(3)
    for max_sub in (1, 3, 8, 1000):
        f = tmp_path / f"m{max_sub}.bin"
        payloads = [rng.bytes(int(n)) for n in (0, 1, 7, 8, 9, 100, 257)]
        for b in payloads:
            assert record_writer.append_fortran_record(str(f).encode(), b, len(b), max_sub) == 0
        assert read_fortran_records(str(f)) == payloads, max_sub
    assert record_writer.append_fortran_record(str(tmp_path / "bad.bin").encode(), b"x", 1, 0) == 1


@pytest.mark.parametrize("edit,what", [("nz=10", "nz=3000000000"), ("nx=1,ny=1,nz=10", "nx=16777216,ny=16777216,nz=4096"),
                                       ("nw=2", "nw=-5")])
def test_deck_refuses_out_of_range_resolution(tmp_path, edit, what):
    """Dimensions beyond int32, beyond the library's 2^56-element block limit, or negative come
    back as OCO_EDIM before anything is allocated."""
    from ocotillo_b200 import OcoError, deck_block_inputs
    d = tmp_path / "agn"
    shutil.copytree(os.path.join(SAMPLES, "NongreyAGN"), d)
    txt = open(d / "resolution.in").read()
    assert edit in txt
    open(d / "resolution.in", "w").write(txt.replace(edit, what))
    with pytest.raises(OcoError) as e:
        deck_block_inputs(str(d))
    assert e.value.code == -10, e.value


def test_run_deck_without_gpu_fails_cleanly(tmp_path):
    """Without a device the deck run reads the deck, creates the output folder and returns the
    context's error code (no exception crosses the C ABI, nothing is left behind but the folder)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from ocotillo_b200 import OcoError, run_deck
    with pytest.raises(OcoError) as e:
        run_deck(os.path.join(SAMPLES, "NongreyAGN"), out_dir=str(tmp_path / "out"))
    assert e.value.code == -5
    assert os.listdir(tmp_path / "out") == []
    d = tmp_path / "agn"
    shutil.copytree(os.path.join(SAMPLES, "NongreyAGN"), d)
    txt = open(d / "resolution.in").read().replace("nz=10", "nz=1")
    open(d / "resolution.in", "w").write(txt)
    with pytest.raises(OcoError) as e:
        run_deck(str(d), out_dir=str(tmp_path / "out2"))
    assert e.value.code == -10


def test_deck_executable_arguments_and_errors(tmp_path):
    """The command-line driver: a bad form or option exits 2 with its usage, a deck that cannot
    be read exits 1 with the library's message, and without a device the run exits 1 after
    reading the deck."""
    import subprocess
    import ocotillo_b200
    exe = os.path.join(os.path.dirname(ocotillo_b200.__file__), "flux_feautrier_b200")
    run = lambda *args: subprocess.run([exe, *args], capture_output=True, text=True, timeout=120)
    r = run("--form", "quad")
    assert r.returncode == 2 and "unknown form quad" in r.stderr
    r = run("--bogus")
    assert r.returncode == 2 and "usage:" in r.stderr
    r = run("--deck", str(tmp_path))
    assert r.returncode == 1 and "resolution.in" in r.stderr
    import torch
    if not torch.cuda.is_available():
        r = run("--deck", os.path.join(SAMPLES, "NongreyAGN"), "--out", str(tmp_path / "out"))
        assert r.returncode == 1 and r.stderr.strip()
