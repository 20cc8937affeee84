"""The mixed-precision form (FP64 Saha; FP32 log-space opacities, difference-form pivots and
back-substitution) against the stable FP64 form of the oracle.

Tolerances (relative, per element): emergent flux V at the top and bottom <= 1e-4 (the target
of the form); kappa <= 3e-5; mean intensity U <= 5e-4.  Interior V is checked relative to the
largest |V| of its item (it changes sign inside the slab), <= 5e-4.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_FLUX, TOL_KAPPA, TOL_U, TOL_VINT = 1e-4, 3e-5, 5e-4, 5e-4


@pytest.fixture(scope="module")
def engine():
    import torch
    assert torch.cuda.is_available()
    from ocotillo_b200 import Engine
    e = Engine(0)
    yield e
    e.close()


def _rel(a, b):
    return np.abs(a - b) / np.abs(b)


def _check(out, ref, what, flux=True):
    assert np.isfinite(out["U"]).all() and np.isfinite(out["V"]).all(), what
    assert _rel(out["kappa"], ref["kappa"]).max() <= TOL_KAPPA, what
    assert _rel(out["U"], ref["U"]).max() <= TOL_U, what
    if not flux:
        return
    assert _rel(out["Vtop"], ref["V"][..., -1]).max() <= TOL_FLUX, what
    assert _rel(out["Vbot"], ref["V"][..., 0]).max() <= TOL_FLUX, what
    vmax = np.abs(ref["V"]).max(axis=-1, keepdims=True)
    assert (np.abs(out["V"] - ref["V"]) / vmax).max() <= TOL_VINT, what


def test_mixed_agn_grid_columns(engine, oracle):
    from ocotillo_b200 import workloads
    rho, T, dz = workloads.agn_block(4, 4, 512, seed=2)
    wa = workloads.log_wavelengths(256)
    engine.set_wavelengths(wa)
    out = engine.solve_block(rho, T, dz, form="mixed")
    ref = oracle.solve_block(rho, T, wa, dz, form=oracle.FORM_STABLE, backend="ocomath")
    _check(out, ref, "agn grid")


def test_mixed_precision_columns(engine, oracle):
    from ocotillo_b200 import workloads
    rho, T, dz, _ = workloads.precision_block(3, 3, 1024, seed=3)
    wa = workloads.log_wavelengths(192)
    engine.set_wavelengths(wa)
    out = engine.solve_block(rho, T, dz, form="mixed")
    ref = oracle.solve_block(rho, T, wa, dz, form=oracle.FORM_STABLE, backend="ocomath")
    _check(out, ref, "precision config")


@pytest.mark.parametrize("nz,nw", [(2, 7), (3, 40), (4, 33), (5, 64), (9, 31)])
def test_mixed_small_sizes(engine, oracle, nz, nw):
    from ocotillo_b200 import workloads
    rho, T, _ = workloads.agn_block(2, 3, nz, seed=nz + 40)
    dz = 2.5e14
    wa = workloads.log_wavelengths(nw, 1000.0, 30000.0)
    engine.set_wavelengths(wa)
    out = engine.solve_block(rho, T, dz, form="mixed")
    ref = oracle.solve_block(rho, T, wa, dz, form=oracle.FORM_STABLE, backend="ocomath")
    # For nz < 4 the ghost zones feed each other and both forms keep the reference's stencil
    # on U, whose differences are below FP64 resolution in these optically thin columns: the
    # flux there is rounding noise in any precision, so only U and kappa are compared.
    _check(out, ref, f"nz={nz} nw={nw}", flux=nz >= 4)


def test_mixed_device_layout_matches_host_path(engine):
    import torch
    from ocotillo_b200 import workloads
    rho, T, dz = workloads.agn_block(3, 5, 64, seed=8)
    wa = workloads.log_wavelengths(96)
    engine.set_wavelengths(wa)
    host = engine.solve_block(rho, T, dz, form="mixed")
    nx, ny, nz = rho.shape
    nw = len(wa)
    dev = torch.device("cuda:0")
    out = {"U": torch.empty((nz + 6, nx * ny, nw), dtype=torch.float64, device=dev),
           "kappa": torch.empty((nz, nx * ny, nw), dtype=torch.float64, device=dev),
           "V": torch.empty((nz, nx * ny, nw), dtype=torch.float64, device=dev)}
    engine.solve_block_device(torch.from_numpy(rho).to(dev), torch.from_numpy(T).to(dev), dz, out, form="mixed",
                              layout=1)
    torch.cuda.synchronize()
    U = out["U"].cpu().numpy().reshape(nz + 6, nx, ny, nw).transpose(3, 1, 2, 0)
    V = out["V"].cpu().numpy().reshape(nz, nx, ny, nw).transpose(3, 1, 2, 0)
    assert np.array_equal(U, host["U"]) and np.array_equal(V, host["V"])


def test_mixed_reference_decks_close(engine, oracle, tmp_path):
    import os
    from conftest import SAMPLES
    for deck in ("NongreyAGN", "ReadFromAthena", "multiInTest"):
        d = tmp_path / deck
        d.mkdir()
        rc, msg = oracle.run_deck(os.path.join(SAMPLES, deck), str(d), backend="ocomath")
        meta = open(d / "inputs_meta.txt").read().split()
        nx, ny, nz, nw = (int(v) for v in meta[:4])
        dz = float(meta[4])
        rho = np.fromfile(d / "inputs_rho.bin").reshape(nx, ny, nz)
        T = np.fromfile(d / "inputs_T.bin").reshape(nx, ny, nz)
        wa = np.fromfile(d / "inputs_wa.bin")
        engine.set_wavelengths(wa)
        out = engine.solve_block(rho, T, dz, form="mixed")
        ref = oracle.solve_block(rho, T, wa, dz, form=oracle.FORM_STABLE, backend="ocomath")
        _check(out, ref, deck)


# Columns of the benchmark AGN grid (workloads.agn_block(256, 256, 512, seed=2), flattened
# index ix*256 + iy) whose emergent flux the FP32 arithmetic resolves worst: a whole-grid study
# of the mixed arithmetic (host build) against the stable FP64 oracle found every item above
# 1e-4 (387 of 1.7e7) in the first 14 of them, up to 9.5e-2 relative.
SENSITIVE_AGN_COLUMNS = [22411, 65490, 22663, 8517, 33061, 12343, 35821, 41899, 48354, 38946, 12625, 57049, 43576,
                         47672, 5644, 43762, 23105, 56717, 16326, 25694, 18418, 19536, 12740, 40457, 29247, 63020,
                         3848, 55435, 34630, 4927, 34386, 17057, 37542, 19643, 53654, 23881, 38023, 48054, 33685,
                         49843]


@pytest.fixture(scope="module")
def sensitive_block():
    """64 columns of the benchmark AGN grid: the 40 most sensitive ones and 24 others."""
    from ocotillo_b200 import workloads
    rho, T, dz = workloads.agn_block(256, 256, 512, seed=2)
    cols = SENSITIVE_AGN_COLUMNS + list(range(1000, 1024))
    rho = np.ascontiguousarray(rho.reshape(-1, 512)[cols].reshape(8, 8, 512))
    T = np.ascontiguousarray(T.reshape(-1, 512)[cols].reshape(8, 8, 512))
    return rho, T, dz, workloads.log_wavelengths(256)


def test_mixed_emergent_flux_on_sensitive_agn_columns(engine, oracle, sensitive_block):
    """The 1e-4 bar on the emergent flux holds on the grid's most sensitive columns: the mixed
    kernels flag the items whose flux condition number exceeds 100 and a second kernel re-solves
    them in FP64."""
    rho, T, dz, wa = sensitive_block
    engine.set_wavelengths(wa)
    engine.set_mixed_repair(100.0)
    engine.mixed_repairs()
    out = engine.solve_block(rho, T, dz, form="mixed", want=("Vtop", "Vbot"))
    repaired = engine.mixed_repairs()
    ref = oracle.solve_block(rho, T, wa, dz, form=oracle.FORM_STABLE, backend="ocomath", want=("V",))
    err = np.maximum(_rel(out["Vtop"], ref["V"][..., -1]), _rel(out["Vbot"], ref["V"][..., 0]))
    assert err.max() <= TOL_FLUX, err.max()
    # 40 of these 64 columns are the grid's most sensitive, so a large share of their items is
    # re-solved (about 0.07% of the whole grid's); the count only has to be positive and bounded
    assert 0 < repaired < 0.5 * err.size, repaired


def test_mixed_repair_is_the_stable_fp64_solve(engine, oracle, sensitive_block):
    """Without the re-solve some items of these columns miss 1e-4; with it, every item it changed
    equals the stable FP64 form bit for bit (U at every z, kappa, V and the emergent fluxes)."""
    rho, T, dz, wa = sensitive_block
    engine.set_wavelengths(wa)
    engine.set_mixed_repair(float("inf"))
    raw = engine.solve_block(rho, T, dz, form="mixed")
    assert engine.mixed_repairs() == 0
    engine.set_mixed_repair(100.0)
    fixed = engine.solve_block(rho, T, dz, form="mixed")
    stable = engine.solve_block(rho, T, dz, form="stable")
    changed = (raw["Vtop"] != fixed["Vtop"]) | (raw["Vbot"] != fixed["Vbot"])
    assert changed.any()
    for key in ("U", "kappa", "V", "Vtop", "Vbot"):
        a, b = fixed[key][changed], stable[key][changed]
        assert np.array_equal(a.view(np.uint64), b.view(np.uint64)), key
    ref = oracle.solve_block(rho, T, wa, dz, form=oracle.FORM_STABLE, backend="ocomath", want=("V",))
    worst_raw = max(_rel(raw["Vtop"], ref["V"][..., -1]).max(), _rel(raw["Vbot"], ref["V"][..., 0]).max())
    assert worst_raw > TOL_FLUX  # the columns are sensitive enough to need the re-solve


def test_mixed_repair_in_device_layout_and_batch(engine, oracle, sensitive_block):
    """The block kernels with lambda-fastest device outputs re-solve the same items as the
    host-array path (same bits); the batch kernels (both tilings) re-solve too and meet 1e-4."""
    import torch
    from ocotillo_b200 import TILING_PACKED, TILING_WARP_COLUMN
    rho, T, dz, wa = sensitive_block
    engine.set_wavelengths(wa)
    engine.set_mixed_repair(100.0)
    host = engine.solve_block(rho, T, dz, form="mixed", want=("Vtop", "Vbot"))
    nx, ny, nz = rho.shape
    nw = len(wa)
    dev = torch.device("cuda:0")
    o = {"Vtop": torch.empty((nw, nx, ny), dtype=torch.float64, device=dev),
         "Vbot": torch.empty((nw, nx, ny), dtype=torch.float64, device=dev)}
    engine.solve_block_device(torch.from_numpy(rho).to(dev), torch.from_numpy(T).to(dev), dz, o, form="mixed",
                              layout=1)
    engine.synchronize()
    assert np.array_equal(o["Vtop"].cpu().numpy(), host["Vtop"])
    assert np.array_equal(o["Vbot"].cpu().numpy(), host["Vbot"])
    ncol = nx * ny
    b = engine.batch(np.full(ncol, nz), np.full(ncol, nw), np.full(ncol, dz), wa, np.zeros(ncol, dtype=np.int64),
                     layout=1, form="mixed")
    rd = torch.from_numpy(rho.reshape(-1)).to(dev)
    Td = torch.from_numpy(T.reshape(-1)).to(dev)
    out = b.alloc(dev)
    b.bind(rd, Td, out)
    ref = oracle.solve_block(rho, T, wa, dz, form=oracle.FORM_STABLE, backend="ocomath", want=("V",))
    rtop = ref["V"][..., -1].reshape(nw, ncol).T
    rbot = ref["V"][..., 0].reshape(nw, ncol).T
    for tiling in (TILING_WARP_COLUMN, TILING_PACKED):
        b.set_tiling(tiling)
        out["Vtop"].fill_(float("nan"))
        out["Vbot"].fill_(float("nan"))
        engine.mixed_repairs()
        b.run()
        b.wait()
        assert engine.mixed_repairs() > 0, tiling
        vt = out["Vtop"].cpu().numpy().reshape(ncol, nw)  # per column, nw values from flux_off
        vb = out["Vbot"].cpu().numpy().reshape(ncol, nw)
        assert max(_rel(vt, rtop).max(), _rel(vb, rbot).max()) <= TOL_FLUX, tiling
    b.close()


def _batch_fluxes(eng, rho, T, dz, wa, tiling):
    """Emergent fluxes (per column, nw values) of the block's columns as a ragged batch of eng."""
    import torch
    nx, ny, nz = rho.shape
    nw, ncol = len(wa), nx * ny
    dev = torch.device("cuda:0")
    b = eng.batch(np.full(ncol, nz), np.full(ncol, nw), np.full(ncol, dz), wa, np.zeros(ncol, dtype=np.int64),
                  layout=1, form="mixed")
    out = b.alloc(dev)
    b.bind(torch.from_numpy(rho.reshape(-1)).to(dev), torch.from_numpy(T.reshape(-1)).to(dev), out)
    b.set_tiling(tiling)
    b.run()
    b.wait()
    res = {k: out[k].cpu().numpy().copy() for k in ("U", "kappa", "V", "Vtop", "Vbot")}
    b.close()
    return res


def test_mixed_repair_beyond_the_slots(engine, sensitive_block, monkeypatch):
    """With the re-solve's slots capped at 32 (OCO_REPAIR_SLOTS, read when a context is created),
    the flagged items beyond them take the one-warp-per-item path; block and batch results equal
    those of a context with all its slots (the stable FP64 form for re-solved items) bit for bit."""
    from ocotillo_b200 import TILING_PACKED, TILING_WARP_COLUMN, Engine
    rho, T, dz, wa = sensitive_block
    monkeypatch.setenv("OCO_REPAIR_SLOTS", "32")
    capped = Engine(0)
    monkeypatch.delenv("OCO_REPAIR_SLOTS")
    try:
        capped.set_wavelengths(wa)
        capped.set_mixed_repair(100.0)
        capped.mixed_repairs()
        a = capped.solve_block(rho, T, dz, form="mixed")
        n = capped.mixed_repairs()
        ab = {t: _batch_fluxes(capped, rho, T, dz, wa, t) for t in (TILING_WARP_COLUMN, TILING_PACKED)}
    finally:
        capped.close()
    assert n > 1000, n  # most of the flagged items go beyond the 32 slots
    engine.set_wavelengths(wa)
    engine.set_mixed_repair(100.0)
    b = engine.solve_block(rho, T, dz, form="mixed")
    for key in ("U", "kappa", "V", "Vtop", "Vbot"):
        assert np.array_equal(a[key].view(np.uint64), b[key].view(np.uint64)), key
    for t in (TILING_WARP_COLUMN, TILING_PACKED):
        bb = _batch_fluxes(engine, rho, T, dz, wa, t)
        for key in ("U", "kappa", "V", "Vtop", "Vbot"):
            assert np.array_equal(ab[t][key].view(np.uint64), bb[key].view(np.uint64)), (t, key)


# Columns of the batching config's construction (workloads.ragged_batch(8192, seed=4)) holding a
# cell where the reference's Saha root 0.5 (sqrt(C^2 + 4C) - C) rounds above 1 in a numpy
# evaluation (C ~ 4e8 .. 7e9 at T ~ 13,000-19,000 K): the neutral fraction is then negative, and
# the reference's opacity terms proportional to it turn negative.
NEGATIVE_NEUTRAL_COLUMNS = [194, 4198, 4795, 5044, 6758, 8159]


def test_mixed_negative_neutral_fraction_columns(engine, oracle):
    """Log-space opacities cannot carry a negative term, so the record kernel flags a column with
    such a cell whole: with the condition-number threshold off, its items are re-solved in FP64
    all or none per column (the GPU's Saha decides which columns, within an ulp of numpy's), at
    least one column is; with the default threshold every emergent flux meets 1e-4."""
    from ocotillo_b200 import workloads
    d = workloads.ragged_batch(ncol=8192, seed=4)
    off = np.concatenate([[0], np.cumsum(d["nz"])])
    whole = 0
    for c in NEGATIVE_NEUTRAL_COLUMNS:
        nz, nw, dz = int(d["nz"][c]), int(d["nw"][c]), float(d["dz"][c])
        rho = np.ascontiguousarray(d["rho"][off[c]:off[c] + nz].reshape(1, 1, nz))
        T = np.ascontiguousarray(d["T"][off[c]:off[c] + nz].reshape(1, 1, nz))
        wa = workloads.log_wavelengths(nw)
        engine.set_wavelengths(wa)
        engine.set_mixed_repair(float("inf"))
        engine.mixed_repairs()
        engine.solve_block(rho, T, dz, form="mixed", want=("Vtop", "Vbot"))
        n = engine.mixed_repairs()
        assert n in (0, nw), (c, n, nw)
        whole += n == nw
        engine.set_mixed_repair(100.0)
        out = engine.solve_block(rho, T, dz, form="mixed", want=("Vtop", "Vbot"))
        ref = oracle.solve_block(rho, T, wa, dz, form=oracle.FORM_STABLE, backend="ocomath", want=("V",))
        err = max(_rel(out["Vtop"], ref["V"][..., -1]).max(), _rel(out["Vbot"], ref["V"][..., 0]).max())
        assert err <= TOL_FLUX, (c, err)
    assert whole >= 1
