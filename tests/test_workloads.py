"""The seeded synthetic workloads the benchmark and the tests run on: every documented range
and distribution holds, and a seed always gives the same arrays."""
import math

import numpy as np


def test_grid_wavelengths_and_temperature():
    from ocotillo_b200 import workloads as W
    z, dz = W.grid(512)
    assert z[0] == W.Z0 and math.isclose(z[-1], W.Z1, rel_tol=1e-12) and dz == (W.Z1 - W.Z0) / 511
    wa = W.log_wavelengths(256)
    assert math.isclose(wa[0], 100.0) and math.isclose(wa[-1], 1e5) and np.all(np.diff(wa) > 0)
    assert np.allclose(np.diff(np.log(wa)), math.log(1e3) / 255)
    assert list(W.log_wavelengths(1)) == [100.0]
    T = W.temperature(z)
    assert T.min() == W.T_FLOOR and T.max() <= W.T_MID and math.isclose(W.temperature(np.zeros(1))[0], W.T_MID)


def test_agn_block_distribution_and_determinism():
    from ocotillo_b200 import workloads as W
    rho, T, dz = W.agn_block(8, 8, 512, seed=2)
    assert rho.shape == T.shape == (8, 8, 512) and rho.flags.c_contiguous and T.flags.c_contiguous
    assert np.all(np.isfinite(rho)) and np.all(rho > 0) and np.all(T >= W.T_FLOOR)
    z, _ = W.grid(512)
    base = np.maximum(W.RHO0 * np.exp(-0.5 * z * z / (W.H * W.H)), W.RHO_FLOOR)
    dex = np.log10(rho / base)
    assert abs(dex.mean()) < 0.01 and abs(dex.std() - 0.3) < 0.01  # 0.3 dex lognormal per cell
    rho2, T2, _ = W.agn_block(8, 8, 512, seed=2)
    assert np.array_equal(rho, rho2) and np.array_equal(T, T2)
    assert not np.array_equal(rho, W.agn_block(8, 8, 512, seed=3)[0])


def test_precision_block_density_range():
    from ocotillo_b200 import workloads as W
    for seed in range(20):
        _, _, _, rho0 = W.precision_block(1, 1, 16, seed=seed)
        assert 1e-11 <= rho0 <= 1e-7


def test_ragged_batch_ranges_and_packing():
    from ocotillo_b200 import workloads as W
    d = W.ragged_batch(ncol=512, seed=4)
    nz, nw = d["nz"], d["nw"]
    assert nz.min() >= 64 and nz.max() <= 2048 and nw.min() >= 32 and nw.max() <= 1024
    assert nz.max() > 1024 and nz.min() < 128  # log-uniform: both decades are reached
    assert len(d["rho"]) == len(d["T"]) == nz.sum() and np.all(d["rho"] > 0) and np.all(d["T"] > 0)
    assert np.all(d["dz"] > 0) and np.all(np.isfinite(d["dz"]))
    for i in range(len(nz)):
        w = d["waves"][d["wave_off"][i]:d["wave_off"][i] + nw[i]]
        assert np.array_equal(w, W.log_wavelengths(int(nw[i])))
    d2 = W.ragged_batch(ncol=512, seed=4)
    assert all(np.array_equal(d[k], d2[k]) for k in d)


def test_serving_stream_ranges():
    from ocotillo_b200 import workloads as W
    jobs = W.serving_stream(200, rate=20.0, seed=5)
    t = [j["arrival_s"] for j in jobs]
    assert t[0] == 0.0 and all(b >= a for a, b in zip(t, t[1:]))
    assert 5.0 < t[-1] < 20.0  # 199 gaps of mean 1/20 s
    for j in jobs:
        assert j["nx"] == j["ny"] and j["nx"] in W.SERVING_SIZES
        assert 128 <= j["nz"] <= 1024 and 64 <= j["nw"] <= 512 and 1e-11 <= j["rho0"] <= 1e-7
