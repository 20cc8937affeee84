"""Epilogues of a solved block on the device: upward/downward intensities (calc_intensity,
auxiliary.f90:80-94) and optical depth with the photosphere index (ReadOcotillo.py:248-293),
bit-identical to the reference's definitions evaluated with numpy on the same outputs."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("layout", [0, 1])
def test_intensities_and_optical_depth(layout):
    import torch
    from ocotillo_b200 import Engine, workloads
    e = Engine(0)
    rho, T, dz = workloads.agn_block(3, 4, 96, seed=17)
    wa = workloads.log_wavelengths(40, 900.0, 40000.0)
    e.set_wavelengths(wa)
    nx, ny, nz = rho.shape
    nw, ncol = len(wa), nx * ny
    dev = torch.device("cuda:0")
    mk = lambda *s: torch.empty(s, dtype=torch.float64, device=dev)
    if layout == 0:
        out = {"U": mk(nw, nx, ny, nz + 6), "kappa": mk(nw, nx, ny, nz), "V": mk(nw, nx, ny, nz)}
    else:
        out = {"U": mk(nz + 6, ncol, nw), "kappa": mk(nz, ncol, nw), "V": mk(nz, ncol, nw)}
    r, t = torch.from_numpy(rho).to(dev), torch.from_numpy(T).to(dev)
    e.solve_block_device(r, t, dz, out, form="stable", layout=layout)
    ip, im, tau = torch.empty_like(out["V"]), torch.empty_like(out["V"]), torch.empty_like(out["V"])
    photo = torch.empty((nw, nx, ny), dtype=torch.int32, device=dev)
    e.intensities_device(out["U"], out["V"], rho.shape, nw, {"Ip": ip, "Im": im}, layout=layout)
    e.optical_depth_device(out["kappa"], r, dz, target_tau=2.0 / 3.0, tau=tau, photo=photo, layout=layout)
    e.synchronize()

    def as_ref(a, ghost=0):  # -> (nw, ncol, nz[+6])
        a = a.cpu().numpy()
        return a.reshape(nw, ncol, -1) if layout == 0 else a.reshape(nz + ghost, ncol, nw).transpose(2, 1, 0)

    U, V, K = as_ref(out["U"], 6), as_ref(out["V"]), as_ref(out["kappa"])
    assert np.array_equal(as_ref(ip), U[..., 3:-3] + V)
    assert np.array_equal(as_ref(im), U[..., 3:-3] - V)
    ref_tau = np.cumsum(K * rho.reshape(ncol, nz)[None] * dz, axis=2)  # calculate_optical_depth
    assert np.array_equal(as_ref(tau), ref_tau)
    reached = ref_tau >= 2.0 / 3.0                                     # find_photosphere
    ref_photo = np.where(reached.any(axis=2), reached.argmax(axis=2), -1)
    assert np.array_equal(photo.cpu().numpy().reshape(nw, ncol), ref_photo)
    e.close()
