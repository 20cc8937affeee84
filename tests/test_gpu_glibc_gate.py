"""The plain form against the oracle built on the C library's math (what the gfortran-built
reference calls: exp, log, log10, pow at continuous_opacity.f90:161, 171, 238, 242, 290-298, 407
and gas_state.f90:58-60), not on the shared ocomath.

The reference's arithmetic is ill-conditioned (the Thomas pivot bet = b - a*gam cancels,
auxiliary.f90:35), so a 1e-12 bar can only hold where the problem itself is stable: the
conditioning mask keeps the (column, wavelength) items whose U (every z) and emergent fluxes
change by less than 1e-14 relative when rho is perturbed by one ulp (a relative 2^-52 N(0,1)
per cell, glibc oracle).  Inside the mask the GPU agrees with oracle(glibc) to 1e-12; everywhere
the finite class and the sign of U, kappa and the emergent fluxes agree."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MASK_SENSITIVITY, TOL_MASK = 1e-14, 1e-12


def _rel(a, b):
    with np.errstate(all="ignore"):
        return np.nan_to_num(np.abs(a - b) / np.abs(b), nan=np.inf)


def gate(gpu, ref, ref_pert):
    """Mask fraction, max relative difference inside the mask, class agreement and the fraction
    of bit-identical items (per item over U, kappa, Vtop, Vbot)."""
    s = np.maximum(_rel(ref_pert["U"], ref["U"]).max(-1),
                   np.maximum(_rel(ref_pert["V"][..., -1], ref["V"][..., -1]),
                              _rel(ref_pert["V"][..., 0], ref["V"][..., 0])))
    mask = s < MASK_SENSITIVITY
    d = np.maximum(np.maximum(_rel(gpu["U"], ref["U"]).max(-1), _rel(gpu["kappa"], ref["kappa"]).max(-1)),
                   np.maximum(_rel(gpu["Vtop"], ref["V"][..., -1]), _rel(gpu["Vbot"], ref["V"][..., 0])))
    cls = True
    for a, b in ((gpu["U"], ref["U"]), (gpu["kappa"], ref["kappa"]), (gpu["Vtop"], ref["V"][..., -1]),
                 (gpu["Vbot"], ref["V"][..., 0])):
        fa, fb = np.isfinite(a), np.isfinite(b)
        cls = cls and np.array_equal(fa, fb) and np.array_equal(np.sign(a[fa]), np.sign(b[fb]))
    return {"items": int(d.size), "in_mask": float(mask.mean()),
            "max_rel_in_mask": float(d[mask].max()) if mask.any() else None, "class_equal": bool(cls),
            "bitwise": float((d == 0).mean())}


def _run(oracle, rho, T, dz, wa):
    from ocotillo_b200 import Engine
    eng = Engine(0)
    eng.set_wavelengths(wa)
    gpu = eng.solve_block(rho, T, dz, form="plain", allow_zero_pivot=True)
    eng.close()
    ref = oracle.solve_block(rho, T, wa, dz, form=oracle.FORM_REFERENCE, backend="glibc")
    rng = np.random.default_rng(7)
    rp = rho * (1.0 + 2.0 ** -52 * rng.standard_normal(rho.shape))
    ref_pert = oracle.solve_block(rp, T, wa, dz, form=oracle.FORM_REFERENCE, backend="glibc")
    return gate(gpu, ref, ref_pert)


def test_plain_matches_glibc_oracle_on_the_mask(oracle):
    """AGN columns with the NongreyAGN deck's density floor (1e-15): part of the items are
    well conditioned, and there the libm difference stays below 1e-12."""
    from ocotillo_b200 import workloads
    rho, T, dz = workloads.agn_block(4, 4, 512, seed=2, rho_floor=1e-15)
    g = _run(oracle, rho, T, dz, workloads.log_wavelengths(256)[::4])
    assert g["class_equal"]
    assert g["in_mask"] > 0.01
    assert g["max_rel_in_mask"] <= TOL_MASK


def test_plain_matches_glibc_oracle_classes_on_the_benchmark_grid(oracle):
    """On the benchmark grid's construction (floor 1e-24) no item is conditioned to 1e-14 under a
    one-ulp perturbation of rho; the finite and sign classes still agree everywhere and most
    items are bit-identical (the libm calls that glibc rounds differently are rare)."""
    from ocotillo_b200 import workloads
    rho, T, dz = workloads.agn_block(4, 4, 512, seed=2)
    g = _run(oracle, rho, T, dz, workloads.log_wavelengths(256)[::4])
    assert g["class_equal"]
    assert g["bitwise"] > 0.5
    if g["in_mask"] > 0:
        assert g["max_rel_in_mask"] <= TOL_MASK
