"""The deck layer (input construction, Ew.d editing, Fortran records) on the CPU, against the
oracle's restatement of the reference's driver: the same bytes for every deck's root-block
inputs, the same text for every formatted value."""
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
