"""The oracle against the reference's own golden vectors.

bin/rt_autotest of the reference runs four sample decks and diffs output/diagnostics.txt
(io.f90:31-46, format (I6, nw(2e15.5))) against samples/<deck>/reference.out.  The oracle
must reproduce each file byte for byte, with either math back-end.
"""
import os

import pytest

from conftest import DECKS, SAMPLES


@pytest.mark.parametrize("backend", ["glibc", "ocomath"])
@pytest.mark.parametrize("deck", DECKS)
def test_oracle_reproduces_reference_out(oracle, tmp_path, deck, backend):
    rc, msg = oracle.run_deck(os.path.join(SAMPLES, deck), str(tmp_path), backend=backend)
    assert rc == 0, msg
    got = open(tmp_path / "diagnostics.txt").read()
    want = open(os.path.join(SAMPLES, deck, "reference.out")).read()
    assert got == want


@pytest.mark.parametrize("v,text", [
    (3188400.0, "    0.31884E+07"),
    (0.4e-24, "    0.40000E-24"),
    (-1.0, "   -0.10000E+01"),
    (0.0, "    0.00000E+00"),
    (1.0070e-108, "    0.10070-107"),
    (9.999996e5, "    0.10000E+07"),
    (1.5e200, "    0.15000+201"),
    (float("inf"), "       Infinity"),
    (float("-inf"), "      -Infinity"),
    (float("nan"), "            NaN"),
])
def test_fortran_e15_5(oracle, v, text):
    # gfortran Ew.d editing: 0.ddddd mantissa; a three-digit exponent drops the 'E'.
    assert oracle.format_e(v) == text


def test_grey_nw_guard(oracle):
    # flux_feautrier.f90:84-87: grey RT with nw /= 1 stops.
    import numpy as np
    r = oracle.solve_block(np.ones((1, 1, 10)), np.full((1, 1, 10), 2000.0), [3000.0, 4000.0], 1e15, lgrey=True)
    assert r["rc"] == -4


def test_linear_wavelength_grid(oracle):
    # calc_wavelength, continuous_opacity.f90:37-62: w0 + (i-1)*(w1-w0)/(nw-1); nw=1 -> w0
    import numpy as np
    assert oracle.calc_wavelength(5000.0, 3000.0, 1)[0] == 3000.0
    wa = oracle.calc_wavelength(5000.0, 3000.0, 5)
    assert list(wa) == [3000.0, 3500.0, 4000.0, 4500.0, 5000.0]
