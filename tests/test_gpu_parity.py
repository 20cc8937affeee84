"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle.

FORM_PLAIN must equal the oracle's ocomath back-end bit for bit: same operation order, no
FMA contraction, the same correctly rounded exp/log/pow on both sides.  FORM_STABLE must
equal the oracle's difference-form solve bit for bit.  The reference decks must reproduce
reference.out text-exactly through the GPU.
"""
import os

import numpy as np
import pytest

from conftest import DECKS, SAMPLES

pytestmark = pytest.mark.gpu


def assert_bitwise(a, b, what=""):
    a = np.asarray(a)
    b = np.asarray(b)
    assert a.shape == b.shape, what
    na, nb = np.isnan(a), np.isnan(b)
    assert np.array_equal(na, nb), f"{what}: NaN pattern differs"
    ua, ub = a[~na].view(np.uint64), b[~nb].view(np.uint64)
    bad = np.count_nonzero(ua != ub)
    assert bad == 0, f"{what}: {bad} of {ua.size} values differ; max rel {np.nanmax(np.abs(a[~na]-b[~nb])/np.abs(b[~nb]))}"


@pytest.fixture(scope="module")
def engine():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    from ocotillo_b200 import Engine
    e = Engine(0)
    yield e
    e.close()


def _deck_inputs(oracle, deck, tmp):
    rc, msg = oracle.run_deck(os.path.join(SAMPLES, deck), str(tmp), backend="ocomath")
    assert rc == 0, msg
    meta = open(tmp / "inputs_meta.txt").read().split()
    nx, ny, nz, nw = (int(v) for v in meta[:4])
    dz, lgrey, sg, fit = float(meta[4]), int(meta[5]), float(meta[6]), float(meta[7])
    rho = np.fromfile(tmp / "inputs_rho.bin").reshape(nx, ny, nz)
    T = np.fromfile(tmp / "inputs_T.bin").reshape(nx, ny, nz)
    wa = np.fromfile(tmp / "inputs_wa.bin")
    return rho, T, wa, dz, bool(lgrey), sg, fit


@pytest.mark.parametrize("deck", DECKS)
def test_reference_decks_through_gpu(engine, oracle, tmp_path, deck):
    rho, T, wa, dz, lgrey, sg, fit = _deck_inputs(oracle, deck, tmp_path)
    if not lgrey:
        engine.set_wavelengths(wa)
    out = engine.solve_block(rho, T, dz, fully_ionized_T=fit, lgrey=lgrey, sigma_grey=sg)
    ref = oracle.solve_block(rho, T, wa, dz, fully_ionized_T=fit, lgrey=lgrey, sigma_grey=sg, backend="ocomath")
    assert ref["rc"] == 0
    for k in ("U", "kappa", "V"):
        assert_bitwise(out[k], ref[k], f"{deck} {k}")
    # diagnostics.txt (io.f90:31-46) of the last column of the block, from GPU results
    nz = rho.shape[2]
    lines = []
    for i in range(nz):
        cells = [oracle.format_e(out["U"][iw, -1, -1, 3 + i]) for iw in range(len(wa))]
        cells += [oracle.format_e(out["kappa"][iw, -1, -1, i]) for iw in range(len(wa))]
        lines.append("%6d" % (i + 1) + "".join(cells) + "\n")
    assert "".join(lines) == open(os.path.join(SAMPLES, deck, "reference.out")).read()


@pytest.mark.parametrize("form", ["plain", "stable"])
def test_synthetic_agn_bitwise(engine, oracle, form):
    from ocotillo_b200 import workloads
    rho, T, dz = workloads.agn_block(5, 3, 96, seed=7)
    wa = workloads.log_wavelengths(40)
    engine.set_wavelengths(wa)
    out = engine.solve_block(rho, T, dz, form=form, allow_zero_pivot=True)
    ref = oracle.solve_block(rho, T, wa, dz, form=oracle.FORM_STABLE if form == "stable" else oracle.FORM_REFERENCE,
                             backend="ocomath")
    assert out["zero_pivot"] == (ref["rc"] == -3)
    for k in ("U", "kappa", "V"):
        assert_bitwise(out[k], ref[k], f"{form} {k}")
    assert_bitwise(out["Vtop"], ref["V"][..., -1], "Vtop")
    assert_bitwise(out["Vbot"], ref["V"][..., 0], "Vbot")


@pytest.mark.parametrize("nz", [2, 3, 4, 5, 7])
def test_small_nz_ghost_order(engine, oracle, nz):
    # For nz < 4 the reference's ghost update reads ghosts it has just written.
    from ocotillo_b200 import workloads
    rho, T, _ = workloads.agn_block(2, 2, nz, seed=nz)
    dz = 3.3e14
    wa = workloads.log_wavelengths(5, 1000.0, 20000.0)
    engine.set_wavelengths(wa)
    out = engine.solve_block(rho, T, dz, allow_zero_pivot=True)
    ref = oracle.solve_block(rho, T, wa, dz, backend="ocomath")
    assert out["zero_pivot"] == (ref["rc"] == -3)
    for k in ("U", "kappa", "V"):
        assert_bitwise(out[k], ref[k], f"nz={nz} {k}")


def test_grey_config(engine, oracle):
    from ocotillo_b200 import workloads
    rho, T, dz = workloads.grey_isothermal()
    out = engine.solve_block(rho, T, dz, lgrey=True, sigma_grey=0.4)
    ref = oracle.solve_block(rho, T, [3000.0], dz, lgrey=True, sigma_grey=0.4, backend="ocomath")
    for k in ("U", "kappa", "V"):
        assert_bitwise(out[k], ref[k], f"grey {k}")


def test_grey_requires_one_wavelength(engine):
    from ocotillo_b200 import OcoError, workloads
    rho, T, dz = workloads.grey_isothermal()
    engine.set_wavelengths([3000.0, 4000.0])
    prm_rc = None
    try:
        engine.lib.oco_solve_block  # noqa
        p = engine.params(rho.shape, 2, dz, lgrey=True)
        import ctypes
        from ocotillo_b200.engine import _ptr
        U = np.empty((2, 1, 1, 16))
        prm_rc = engine.lib.oco_solve_block(engine.ctx, ctypes.byref(p), _ptr(np.ascontiguousarray(rho)),
                                            _ptr(np.ascontiguousarray(T)), _ptr(U), None, None, None, None)
    except OcoError:
        pass
    assert prm_rc == -4


@pytest.mark.parametrize("layout", [0, 1])
def test_device_entry_layouts(engine, layout):
    import torch
    from ocotillo_b200 import workloads
    rho, T, dz = workloads.agn_block(3, 4, 40, seed=3)
    wa = workloads.log_wavelengths(33)
    engine.set_wavelengths(wa)
    host = engine.solve_block(rho, T, dz, allow_zero_pivot=True)
    nx, ny, nz = rho.shape
    nw = len(wa)
    dev = torch.device("cuda:0")
    if layout == 0:
        shp = {"U": (nw, nx, ny, nz + 6), "kappa": (nw, nx, ny, nz), "V": (nw, nx, ny, nz)}
    else:
        shp = {"U": (nz + 6, nx * ny, nw), "kappa": (nz, nx * ny, nw), "V": (nz, nx * ny, nw)}
    out = {k: torch.full(s, float("nan"), dtype=torch.float64, device=dev) for k, s in shp.items()}
    out["Vtop"] = torch.empty((nw, nx, ny), dtype=torch.float64, device=dev)
    out["Vbot"] = torch.empty((nw, nx, ny), dtype=torch.float64, device=dev)
    engine.solve_block_device(torch.from_numpy(rho).to(dev), torch.from_numpy(T).to(dev), dz, out, layout=layout)
    torch.cuda.synchronize()
    try:
        engine.synchronize()
    except Exception as e:
        assert getattr(e, "code", None) == -3
    got = {k: v.cpu().numpy() for k, v in out.items()}
    if layout == 1:
        got["U"] = got["U"].reshape(nz + 6, nx, ny, nw).transpose(3, 1, 2, 0)
        got["kappa"] = got["kappa"].reshape(nz, nx, ny, nw).transpose(3, 1, 2, 0)
        got["V"] = got["V"].reshape(nz, nx, ny, nw).transpose(3, 1, 2, 0)
    for k in ("U", "kappa", "V", "Vtop", "Vbot"):
        assert_bitwise(np.ascontiguousarray(got[k]), host[k], f"layout {layout} {k}")


def test_chunked_solve_matches_single_chunk(engine, monkeypatch):
    # The host path runs in column chunks; results cannot depend on the chunking.
    from ocotillo_b200 import Engine, workloads
    rho, T, dz = workloads.agn_block(7, 5, 48, seed=9)
    wa = workloads.log_wavelengths(17)
    engine.set_wavelengths(wa)
    a = engine.solve_block(rho, T, dz, allow_zero_pivot=True)
    monkeypatch.setenv("OCO_WORKSPACE_GB", "0.0005")
    small = Engine(0)
    small.set_wavelengths(wa)
    b = small.solve_block(rho, T, dz, allow_zero_pivot=True)
    small.close()
    for k in ("U", "kappa", "V", "Vtop", "Vbot"):
        assert_bitwise(a[k], b[k], k)


def test_device_entry_alternating_streams(engine, oracle):
    """Device-array calls share the context's records, scratch and layout temporaries: a call
    on another stream than the pending one is ordered after it on the device, so calls
    alternating between two streams each give the oracle's bits."""
    import torch
    from ocotillo_b200 import workloads
    rho, T, dz = workloads.agn_block(16, 16, 128, seed=23)
    wa = workloads.log_wavelengths(64)
    engine.set_wavelengths(wa)
    nx, ny, nz = rho.shape
    nw = len(wa)
    dev = torch.device("cuda:0")
    r, t = torch.from_numpy(rho).to(dev), torch.from_numpy(T).to(dev)
    mk = lambda *s: torch.full(s, float("nan"), dtype=torch.float64, device=dev)
    outs = [{"U": mk(nw, nx, ny, nz + 6), "V": mk(nw, nx, ny, nz)} for _ in range(4)]
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    torch.cuda.synchronize()
    for i, o in enumerate(outs):
        engine.solve_block_device(r, t, dz, o, form="stable", layout=0, stream=s1 if i % 2 == 0 else s2)
    torch.cuda.synchronize()
    engine.synchronize()
    ref = oracle.solve_block(rho, T, wa, dz, form=oracle.FORM_STABLE, backend="ocomath")
    for i, o in enumerate(outs):
        assert_bitwise(o["U"].cpu().numpy(), ref["U"], f"call {i} U")
        assert_bitwise(o["V"].cpu().numpy(), ref["V"], f"call {i} V")
