"""Serving loop (oco_server_*): admission by slots and device footprint, overlapping jobs, and
results that do not depend on the mix.

Invariance: every job's results in a mix of concurrent jobs (small launches, so the jobs'
launches interleave and run side by side with reduced grids) are bit-for-bit those of the same
job solved alone through the block solve (host arrays): each (column, wavelength) item runs
the same arithmetic whatever grid and stream run it.
"""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    import torch
    assert torch.cuda.is_available()
    from ocotillo_b200 import Engine
    e = Engine(0)
    yield e
    e.close()


def _job(seed, nx, ny, nz, nw):
    from ocotillo_b200 import workloads
    rho, T, dz, _ = workloads.precision_block(nx, ny, nz, seed=seed)
    wa = workloads.log_wavelengths(nw)
    return rho, T, dz, wa


JOBS = [  # (seed, nx, ny, nz, nw, form, want_fields)
    (31, 8, 8, 128, 64, "mixed", True),
    (32, 16, 8, 200, 96, "plain", False),
    (33, 4, 4, 300, 33, "stable", True),
    (34, 12, 12, 128, 80, "mixed", False),
    (35, 8, 4, 64, 40, "plain", True),
    (36, 10, 10, 150, 128, "mixed", False),
]


def test_server_results_same_alone_and_in_the_mix(engine):
    import torch
    from ocotillo_b200 import Server
    srv = Server(0, max_jobs=3, max_nz=512, chunk_points=1 << 16)
    dev = torch.device("cuda:0")
    ids, inputs = [], []
    for k, (seed, nx, ny, nz, nw, form, fields) in enumerate(JOBS):
        rho, T, dz, wa = _job(seed, nx, ny, nz, nw)
        if k % 2:  # device inputs for half of the jobs
            r, t = torch.from_numpy(rho).to(dev), torch.from_numpy(T).to(dev)
        else:
            r, t = rho, T
        ids.append(srv.submit(r, t, wa, dz, form=form, want_fields=fields))
        inputs.append((rho, T, dz, wa, form, fields))
    got = []
    for jid in ids:
        srv.wait(jid, 120.0)
        st = srv.status(jid)
        assert st["state"] == "done" and st["inputs_consumed"]
        assert st["submit_s"] <= st["admit_s"] <= st["done_s"]
        got.append(srv.fetch(jid))
    srv.close()
    for (rho, T, dz, wa, form, fields), out in zip(inputs, got):
        engine.set_wavelengths(wa)
        ref = engine.solve_block(rho, T, dz, form=form, allow_zero_pivot=True)
        for k in ("Vtop", "Vbot") + (("U", "kappa", "V") if fields else ()):
            assert np.array_equal(out[k], ref[k], equal_nan=True), (form, k)
        assert ("U" in out) == fields


def test_server_jobs_overlap_and_admission_waits_for_memory():
    from ocotillo_b200 import Server
    rho, T, dz, wa = _job(41, 32, 32, 256, 128)
    ncol, nz, nw = 32 * 32, 256, 128
    # footprint of one job that keeps its fields: inputs (released when it finishes) and results
    jb = 2 * rho.nbytes + 8 * ncol * nw * (2 + (nz + 6) + 2 * nz)
    # two slots, memory for two and a half jobs: the first two are admitted at once and run
    # side by side; the third waits until a fetch returns the results' memory
    srv = Server(0, max_jobs=2, max_nz=256, budget_bytes=2.5 * jb, chunk_points=1 << 18)
    ids = [srv.submit(rho, T, wa, dz, form="plain", want_fields=True) for _ in range(3)]
    for j in ids[:2]:
        srv.wait(j, 120.0)
    s = [srv.status(j) for j in ids]
    assert max(s[0]["admit_s"], s[1]["admit_s"]) < min(s[0]["done_s"], s[1]["done_s"])
    time.sleep(0.05)
    assert srv.status(ids[2])["state"] == "queued"
    r0 = srv.fetch(ids[0])
    srv.wait(ids[2], 120.0)
    assert srv.status(ids[2])["admit_s"] >= s[1]["done_s"]
    r2 = srv.fetch(ids[2])
    for k in ("Vtop", "U", "V"):
        assert np.array_equal(r0[k], r2[k], equal_nan=True), k
    srv.fetch(ids[1])
    srv.close()


def test_server_rejects_and_shuts_down():
    from ocotillo_b200 import OcoError, Server
    rho, T, dz, wa = _job(42, 8, 8, 64, 32)
    srv = Server(0, max_jobs=1, budget_bytes=float(rho.nbytes), chunk_points=1 << 16)
    with pytest.raises(OcoError) as e:
        srv.submit(rho, T, wa, dz)  # footprint above the budget: never admissible
    assert e.value.code == -8
    bad_wa = wa.copy()
    bad_wa[3] = float("nan")
    with pytest.raises(OcoError) as e:
        srv.submit(rho, T, bad_wa, dz)  # refused at submission, not failed later
    assert e.value.code == -1 and "wavelength 3" in str(e.value)
    with pytest.raises(OcoError) as e:
        srv.submit(rho, T, wa, float("inf"))
    assert e.value.code == -1
    srv.close()
    # shutting down with one job running and three queued: the queued ones are dropped, the
    # running one finishes, and the call returns
    srv = Server(0, max_jobs=1, chunk_points=1 << 14)
    big = _job(43, 64, 64, 256, 128)
    for _ in range(4):
        srv.submit(big[0], big[1], big[3], big[2], form="plain")
    t0 = time.time()
    srv.close()
    assert time.time() - t0 < 60.0
