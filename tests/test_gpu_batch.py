"""Ragged batches (oco_batch_*): independent columns of different nz, dz and wavelength grids
in one persistent launch replayed as a CUDA graph.

Mixed form: per column the batch runs the arithmetic of the block solve's mixed form (the
batch kernels keep their Thomas scratch in 12-byte records, the block kernels in float4 ones,
holding the same values), so every column must equal a 1x1 block solve of it bit for bit; a
few columns are also compared with the stable FP64 oracle at the mixed form's tolerances.
Tilings and graph replays must give identical results.

Plain and stable FP64 forms: per item the block solve's FP64 arithmetic, so every column must
equal a 1x1 block solve of it bit for bit, and the plain form must equal the oracle (reference
arithmetic, ocomath back-end) bit for bit.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_FLUX, TOL_KAPPA, TOL_U = 1e-4, 3e-5, 5e-4


@pytest.fixture(scope="module")
def engine():
    import torch
    assert torch.cuda.is_available()
    from ocotillo_b200 import Engine
    e = Engine(0)
    yield e
    e.close()


def _small_batch(seed=11):
    """Columns covering the edge sizes: nz 2..300 (2 and 3 take the short-column path), nw 1..97
    (partial 32-wavelength tiles), several grids shared between columns."""
    from ocotillo_b200 import workloads
    rng = np.random.default_rng(seed)
    nz = np.array([2, 3, 4, 5, 7, 31, 32, 33, 64, 100, 257, 300, 40, 41, 64, 2, 128, 90], dtype=np.int64)
    nw = np.array([1, 5, 31, 32, 33, 64, 70, 97, 1, 7, 40, 33, 32, 64, 96, 3, 65, 31], dtype=np.int64)
    grids, waves, off = {}, [], []
    pos = 0
    for w in nw:
        w = int(w)
        if w not in grids:
            grids[w] = pos
            waves.append(workloads.log_wavelengths(w, 900.0, 40000.0))
            pos += w
        off.append(grids[w])
    rhos, Ts, dzs = [], [], []
    for n in nz:
        r, t, dz = workloads.athena_column(int(n), rng, sigma_dex=0.3)
        rhos.append(r)
        Ts.append(t)
        dzs.append(dz)
    return {"nz": nz, "nw": nw, "dz": np.array(dzs), "wave_off": np.array(off), "waves": np.concatenate(waves),
            "rho": np.concatenate(rhos), "T": np.concatenate(Ts)}


def _make(engine, d, layout, form="mixed"):
    import torch
    b = engine.batch(d["nz"], d["nw"], d["dz"], d["waves"], d["wave_off"], layout=layout, form=form)
    dev = torch.device("cuda:0")
    rho = torch.from_numpy(d["rho"]).to(dev)
    T = torch.from_numpy(d["T"]).to(dev)
    out = b.alloc(dev)
    b.bind(rho, T, out)
    return b, rho, T, out


def _block(engine, d, i, form="mixed"):
    """Column i as a 1x1 block through the block solve (host arrays)."""
    o = np.concatenate([[0], np.cumsum(d["nz"])])
    nz, nw = int(d["nz"][i]), int(d["nw"][i])
    wa = d["waves"][d["wave_off"][i]:d["wave_off"][i] + nw]
    engine.set_wavelengths(wa)
    rho = d["rho"][o[i]:o[i + 1]].reshape(1, 1, nz)
    T = d["T"][o[i]:o[i + 1]].reshape(1, 1, nz)
    return engine.solve_block(rho, T, float(d["dz"][i]), form=form, allow_zero_pivot=True), rho, T, wa


def _same(t, ref):
    """Bit-for-bit equality; the reference arithmetic can give NaN (a zero pivot), which must
    then sit in the same places."""
    a = np.ascontiguousarray(t.cpu().numpy() if hasattr(t, "cpu") else t)
    ref = np.ascontiguousarray(ref)
    return a.shape == ref.shape and np.array_equal(a.view(np.uint64), ref.view(np.uint64))


def _run_fp64(b):
    """Runs a plain/stable batch; a zero pivot (plain form) is reported after every item is done."""
    from ocotillo_b200 import OcoError
    b.run()
    try:
        b.wait()
    except OcoError as e:
        assert e.code == -3, e


def _rel(a, b):
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300)))


@pytest.mark.parametrize("layout", [0, 1])
def test_batch_matches_block_solve(engine, layout):
    d = _small_batch()
    b, _, _, out = _make(engine, d, layout)
    b.run()
    b.wait()
    for i in range(len(d["nz"])):
        ref, _, _, _ = _block(engine, d, i)
        U = b.column(out, i, "U").cpu().numpy()         # (nz+6, nw)
        K = b.column(out, i, "kappa").cpu().numpy()
        V = b.column(out, i, "V").cpu().numpy()
        vt = b.column(out, i, "Vtop").cpu().numpy()
        vb = b.column(out, i, "Vbot").cpu().numpy()
        what = f"column {i} nz={d['nz'][i]} nw={d['nw'][i]} layout={layout}"
        # the same arithmetic per item (the batch kernels keep 12-byte scratch records, the
        # block kernels float4 ones, which hold the same values): bit for bit
        assert _same(U, ref["U"][:, 0, 0, :].T), what
        assert _same(K, ref["kappa"][:, 0, 0, :].T), what
        assert _same(V, ref["V"][:, 0, 0, :].T), what
        assert np.array_equal(vt, V[-1]) and np.array_equal(vb, V[0]), what
    b.close()


def test_batch_tilings_and_replay_identical(engine):
    d = _small_batch(seed=12)
    b, rho, T, out = _make(engine, d, 1)
    results = []
    for tiling, bps in (("warp_column", 0), ("packed", 0), ("warp_column", 2), ("packed", 1)):
        b.set_tiling(tiling, bps)
        for _ in range(2):  # graph replay twice
            for v in out.values():
                v.fill_(float("nan"))
            b.run()
            b.wait()
            results.append({k: v.cpu().numpy().copy() for k, v in out.items()})
    for r in results[1:]:
        for k in r:
            assert np.array_equal(r[k], results[0][k]), k
    info = b.info()
    assert info["graph_launches"] == 8 and info["npoints"] == int((d["nz"] * d["nw"]).sum())
    b.close()


def test_batch_tune_keeps_results(engine):
    d = _small_batch(seed=13)
    b, rho, T, out = _make(engine, d, 1)
    b.run()
    b.wait()
    first = {k: v.cpu().numpy().copy() for k, v in out.items()}
    info = b.tune()
    assert info["tuned"]
    assert len(info["candidates"]) >= 2 and all(c["ms"] > 0 for c in info["candidates"])
    best = min(info["candidates"], key=lambda c: c["ms"])
    assert (info["tiling"], info["blocks_per_sm"]) == (best["tiling"], best["blocks_per_sm"])
    for v in out.values():
        v.zero_()
    b.run()
    b.wait()
    for k, v in out.items():
        assert np.array_equal(v.cpu().numpy(), first[k]), k
    b.close()


def test_batch_rebinding_new_inputs(engine):
    """In-place new input values are picked up by the replayed graph; rebinding to other
    arrays recaptures."""
    d = _small_batch(seed=14)
    b, rho, T, out = _make(engine, d, 1)
    b.run()
    b.wait()
    U1 = out["U"].cpu().numpy().copy()
    T.mul_(1.05)
    b.run()
    b.wait()
    U2 = out["U"].cpu().numpy().copy()
    assert not np.array_equal(U1, U2)
    d2 = dict(d, T=d["T"] * 1.05)
    b2, _, _, out2 = _make(engine, d2, 1)
    b2.run()
    b2.wait()
    assert np.array_equal(out2["U"].cpu().numpy(), U2)
    b.close()
    b2.close()


def test_batch_against_oracle(engine, oracle):
    d = _small_batch(seed=15)
    b, _, _, out = _make(engine, d, 0)
    b.run()
    b.wait()
    o = np.concatenate([[0], np.cumsum(d["nz"])])
    for i in range(len(d["nz"])):
        nz, nw = int(d["nz"][i]), int(d["nw"][i])
        wa = d["waves"][d["wave_off"][i]:d["wave_off"][i] + nw]
        rho = d["rho"][o[i]:o[i + 1]].reshape(1, 1, nz)
        T = d["T"][o[i]:o[i + 1]].reshape(1, 1, nz)
        ref = oracle.solve_block(rho, T, wa, float(d["dz"][i]), form=oracle.FORM_STABLE, backend="ocomath")
        what = f"column {i} nz={nz} nw={nw}"
        assert _rel(b.column(out, i, "kappa").cpu().numpy(), ref["kappa"][:, 0, 0, :].T) <= TOL_KAPPA, what
        assert _rel(b.column(out, i, "U").cpu().numpy(), ref["U"][:, 0, 0, :].T) <= TOL_U, what
        if nz >= 4:  # see test_gpu_mixed.test_mixed_small_sizes for nz < 4
            assert _rel(b.column(out, i, "Vtop").cpu().numpy(), ref["V"][:, 0, 0, -1]) <= TOL_FLUX, what
            assert _rel(b.column(out, i, "Vbot").cpu().numpy(), ref["V"][:, 0, 0, 0]) <= TOL_FLUX, what
    b.close()


def test_batch_rejects_bad_descriptors(engine):
    import torch
    from ocotillo_b200 import OcoError
    d = _small_batch()
    with pytest.raises(OcoError):
        engine.batch(d["nz"], d["nw"], d["dz"], d["waves"], d["wave_off"], form=7)
    bp = engine.batch(d["nz"], d["nw"], d["dz"], d["waves"], d["wave_off"], form="plain")
    with pytest.raises(OcoError):
        bp.set_tiling("packed", 0)  # the packed tiling runs the mixed form only
    bp.close()
    bad = d["nz"].copy()
    bad[3] = 1
    with pytest.raises(OcoError):
        engine.batch(bad, d["nw"], d["dz"], d["waves"], d["wave_off"])
    off = d["wave_off"].copy()
    off[0] = len(d["waves"])
    with pytest.raises(OcoError):
        engine.batch(d["nz"], d["nw"], d["dz"], d["waves"], off)
    b = engine.batch(d["nz"], d["nw"], d["dz"], d["waves"], d["wave_off"])
    dev = torch.device("cuda:0")
    out = b.alloc(dev)
    short = torch.zeros(int(d["nz"].sum()) - 1, dtype=torch.float64, device=dev)
    with pytest.raises(OcoError):
        b.bind(short, short, out)
    with pytest.raises(OcoError):
        b.run()  # not bound
    with pytest.raises(OcoError):
        b.set_tiling("packed", 99)
    b.close()


def test_batch_caller_offsets_and_overlap(engine):
    """A caller's packing (columns in reverse order, NaN-filled gaps between them) gives every
    column the bits of the dense packing; an output family whose column ranges overlap is
    refused at bind when that array is bound, and accepted when it is not."""
    import torch
    from ocotillo_b200 import OcoError, dense_batch_offsets, LAYOUT_LAMBDA_FASTEST
    d = _small_batch(seed=12)
    nz, nw = d["nz"], d["nw"]
    n = len(nz)
    dense = dense_batch_offsets(nz, nw)
    sizes = {"in_off": nz, "u_off": (nz + 6) * nw, "kv_off": nz * nw, "flux_off": nw}
    off = {}
    for k, s in sizes.items():
        pos, o = 3, np.zeros(n, dtype=np.int64)
        for i in reversed(range(n)):
            o[i] = pos
            pos += int(s[i]) + 5
        off[k] = o
    ref, _, _, out0 = _make(engine, d, LAYOUT_LAMBDA_FASTEST, form="plain")
    _run_fp64(ref)

    b = engine.batch(nz, nw, d["dz"], d["waves"], d["wave_off"], form="plain", offsets=off)
    rho = np.full(b.offsets["n_in"], np.nan)
    T = np.full(b.offsets["n_in"], np.nan)
    for i in range(n):
        src, dst = int(dense["in_off"][i]), int(off["in_off"][i])
        rho[dst:dst + nz[i]] = d["rho"][src:src + nz[i]]
        T[dst:dst + nz[i]] = d["T"][src:src + nz[i]]
    dev = torch.device("cuda:0")
    rho, T = torch.from_numpy(rho).to(dev), torch.from_numpy(T).to(dev)
    out = b.alloc(dev)
    b.bind(rho, T, out)
    _run_fp64(b)
    for i in range(n):
        for name in ("U", "kappa", "V", "Vtop", "Vbot"):
            assert _same(b.column(out, i, name), ref.column(out0, i, name).cpu().numpy()), (i, name)
    b.close()

    bad = {k: v.copy() for k, v in off.items()}
    bad["u_off"][4] = bad["u_off"][5] + 1  # column 4's U range starts inside column 5's
    bo = engine.batch(nz, nw, d["dz"], d["waves"], d["wave_off"], form="plain", offsets=bad)
    with pytest.raises(OcoError) as e:
        bo.bind(rho, T, bo.alloc(dev))
    assert "columns 4 and 5 have overlapping U ranges" in str(e.value)
    part = bo.alloc(dev, want=("kappa", "V", "Vtop", "Vbot"))
    bo.bind(rho, T, part)
    _run_fp64(bo)
    for i in range(n):
        for name in ("kappa", "V", "Vtop", "Vbot"):
            assert _same(bo.column(part, i, name), ref.column(out0, i, name).cpu().numpy()), (i, name)
    bo.close()
    ref.close()


def test_batch_replays_alternating_streams(engine):
    """Replays share the batch's work queue: one on another stream than the pending one is
    ordered after it on the device, and every replay gives the same bits."""
    import torch
    d = _small_batch(seed=13)
    b, _, _, out = _make(engine, d, 0, form="plain")
    _run_fp64(b)
    ref = {k: v.cpu().numpy().copy() for k, v in out.items()}
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    for k in out:
        out[k].fill_(float("nan"))
    torch.cuda.synchronize()
    for _ in range(3):
        b.run(stream=s1)
        b.run(stream=s2)
    _run_fp64(b)
    torch.cuda.synchronize()
    for k in out:
        assert _same(out[k], ref[k]), k
    b.close()


@pytest.mark.parametrize("form,layout", [("plain", 0), ("plain", 1), ("stable", 0), ("stable", 1)])
def test_batch_fp64_bitwise_block_solve(engine, form, layout):
    d = _small_batch(seed=16)
    b, _, _, out = _make(engine, d, layout, form=form)
    _run_fp64(b)
    for i in range(len(d["nz"])):
        ref, _, _, _ = _block(engine, d, i, form=form)
        what = f"column {i} nz={d['nz'][i]} nw={d['nw'][i]} form={form} layout={layout}"
        assert _same(b.column(out, i, "U"), ref["U"][:, 0, 0, :].T), what
        assert _same(b.column(out, i, "kappa"), ref["kappa"][:, 0, 0, :].T), what
        assert _same(b.column(out, i, "V"), ref["V"][:, 0, 0, :].T), what
        assert _same(b.column(out, i, "Vtop"), ref["Vtop"][:, 0, 0]), what
        assert _same(b.column(out, i, "Vbot"), ref["Vbot"][:, 0, 0]), what
    b.close()


def test_batch_plain_bitwise_oracle(engine, oracle):
    d = _small_batch(seed=17)
    b, _, _, out = _make(engine, d, 1, form="plain")
    _run_fp64(b)
    b.set_tiling("warp_column", 2)  # another resident-block count, same bits
    first = {k: v.cpu().numpy().copy() for k, v in out.items()}
    _run_fp64(b)
    o = np.concatenate([[0], np.cumsum(d["nz"])])
    for i in range(len(d["nz"])):
        nz, nw = int(d["nz"][i]), int(d["nw"][i])
        wa = d["waves"][d["wave_off"][i]:d["wave_off"][i] + nw]
        rho = d["rho"][o[i]:o[i + 1]].reshape(1, 1, nz)
        T = d["T"][o[i]:o[i + 1]].reshape(1, 1, nz)
        ref = oracle.solve_block(rho, T, wa, float(d["dz"][i]), form=oracle.FORM_REFERENCE, backend="ocomath")
        what = f"column {i} nz={nz} nw={nw}"
        for name in ("U", "kappa", "V"):
            assert _same(b.column(out, i, name), ref[name][:, 0, 0, :].T), (name, what)
    for k, v in out.items():
        assert _same(v, first[k]), k
    b.close()


def test_mixed_batch_refuses_more_items_than_32_bit_slots(engine):
    """The mixed form's FP64 re-solve indexes a batch's flagged items with 32-bit slots, so a
    mixed batch of 2^31 or more (column, wavelength) items is refused at creation (before any
    device allocation); the FP64 forms have no such limit."""
    from ocotillo_b200 import OcoError
    ncol, nw = (1 << 21) + 1, 1024  # 2^31 + 1024 items
    wa = np.geomspace(100.0, 1e5, nw)
    with pytest.raises(OcoError) as e:
        engine.batch(np.full(ncol, 2), np.full(ncol, nw), np.full(ncol, 1e10), wa, np.zeros(ncol, dtype=np.int64),
                     layout=1, form="mixed")
    assert e.value.code == -1 and "2^31-1" in str(e.value)
