"""The deck driver on the GPU: the four reference sample decks through oco_run_deck (and the
flux_feautrier_b200 executable), diagnostics.txt text-identical to the reference's golden
output, the per-block Fortran unformatted files equal to a block solve."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import DECKS, SAMPLES

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("deck", DECKS)
def test_deck_diagnostics_match_golden(tmp_path, deck):
    from ocotillo_b200 import run_deck
    out = tmp_path / "output"
    rc = run_deck(os.path.join(SAMPLES, deck), out_dir=str(out), form="plain")
    assert rc == 0
    got = open(out / "diagnostics.txt").read()
    assert got == open(os.path.join(SAMPLES, deck, "reference.out")).read()
    for f in ("zgrid.txt", "zgrid.bin", "wavegrid.txt", "wavegrid.bin"):
        assert (out / f).exists()


def test_deck_binary_outputs_are_block_solves(tmp_path):
    """multiInTest: 2 x 1 processor blocks, each written as three Fortran records."""
    from ocotillo_b200 import Engine, deck_block_inputs, read_fortran_records, run_deck
    deck = os.path.join(SAMPLES, "multiInTest")
    out = tmp_path / "output"
    assert run_deck(deck, out_dir=str(out), form="plain") == 0
    eng = Engine(0)
    z = np.frombuffer(read_fortran_records(str(out / "zgrid.bin"))[0])
    for ipx in range(2):
        d = deck_block_inputs(deck, iprocx=ipx)
        assert np.array_equal(z, d["z"])
        eng.set_wavelengths(d["wa"])
        ref = eng.solve_block(d["rho"], d["T"], d["dz"], fully_ionized_T=d["fully_ionized_T"])
        bd = out / f"procx{ipx}_procy0"
        for name, key in (("mean_intensity", "U"), ("absorption_coefficients", "kappa"), ("flux", "V")):
            recs = read_fortran_records(str(bd / f"{name}_0000.bin"))
            assert len(recs) == 1
            assert np.array_equal(np.frombuffer(recs[0]), ref[key].ravel()), (ipx, name)
    eng.close()


def test_deck_executable(tmp_path):
    from ocotillo_b200 import engine
    exe = os.path.join(os.path.dirname(engine.__file__), "flux_feautrier_b200")
    deck = tmp_path / "deck"
    shutil.copytree(os.path.join(SAMPLES, "ReadFromAthena"), deck)
    r = subprocess.run([exe, "0000", "--no-binary"], cwd=deck, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert "snapshot: 0000" in r.stdout
    assert open(deck / "output" / "diagnostics.txt").read() == open(deck / "reference.out").read()
    r = subprocess.run([exe, "0000", "--form", "mixed", "--out", str(tmp_path / "mixed")], cwd=deck,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert (tmp_path / "mixed" / "procx0_procy0" / "flux_0000.bin").exists()
