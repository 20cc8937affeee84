"""Failure detection on the GPU without a GPU fault: a bounded wait that runs out is reported
as OCO_ETIMEDOUT and the context stays usable (the next solve is bit-for-bit correct)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_bounded_wait_runs_out_and_context_survives(oracle):
    from ocotillo_b200 import Engine, workloads
    e = Engine(0)
    rc = e.check_bounded_wait(100)
    assert rc == -6, rc
    assert b"bounded wait" in e.lib.oco_last_error(e.ctx)
    # the context keeps working: a staged solve (nw >= 64) after the timeout
    rho, T, dz = workloads.agn_block(2, 2, 64, seed=21)
    wa = workloads.log_wavelengths(64, 2000.0, 20000.0)
    e.set_wavelengths(wa)
    out = e.solve_block(rho, T, dz, form="stable")
    ref = oracle.solve_block(rho, T, wa, dz, form=oracle.FORM_STABLE, backend="ocomath")
    assert np.array_equal(out["U"], ref["U"]) and np.array_equal(out["V"], ref["V"])
    assert e.check_bounded_wait(100) == -6
    e.close()


def test_invalid_arguments_are_refused_and_context_survives(oracle):
    """A non-finite dz, a non-positive wavelength and a wavelength count that does not match
    the tables come back as error codes (nothing launched), and the context keeps working."""
    from ocotillo_b200 import Engine, OcoError, workloads
    e = Engine(0)
    rho, T, dz = workloads.agn_block(2, 2, 32, seed=22)
    wa = workloads.log_wavelengths(8, 2000.0, 20000.0)
    e.set_wavelengths(wa)
    for bad in (float("inf"), float("nan"), -dz, 0.0):
        with pytest.raises(OcoError) as err:
            e.solve_block(rho, T, bad, form="plain")
        assert err.value.code == -1, bad
    bad_wa = wa.copy()
    bad_wa[3] = -bad_wa[3]
    with pytest.raises(OcoError) as err:
        e.set_wavelengths(bad_wa)
    assert err.value.code == -1
    e.set_wavelengths(wa)
    out = e.solve_block(rho, T, dz, form="plain", allow_zero_pivot=True)
    ref = oracle.solve_block(rho, T, wa, dz, form=oracle.FORM_REFERENCE, backend="ocomath")
    assert np.array_equal(out["V"], ref["V"], equal_nan=True)
    e.close()
