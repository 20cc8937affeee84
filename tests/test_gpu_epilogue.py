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


def test_integrated_flux():
    """Wavelength-integrated emergent flux: the trapezoid rule over the wavelength grid (cm) of
    the Vtop plane, against numpy's trapezoid on the same plane (summation orders differ, so
    1e-13 relative)."""
    import torch
    from ocotillo_b200 import Engine, OcoError, workloads
    e = Engine(0)
    rho, T, dz = workloads.agn_block(5, 7, 64, seed=18)
    wa = workloads.log_wavelengths(97)
    e.set_wavelengths(wa)
    nx, ny, nz = rho.shape
    dev = torch.device("cuda:0")
    vt = torch.empty((len(wa), nx, ny), dtype=torch.float64, device=dev)
    r, t = torch.from_numpy(rho).to(dev), torch.from_numpy(T).to(dev)
    e.solve_block_device(r, t, dz, {"Vtop": vt}, form="mixed", layout=0)
    F = e.integrated_flux_device(vt, (nx, ny))
    e.synchronize()
    v = vt.cpu().numpy()
    ref = np.trapezoid(v, x=wa * 1e-8, axis=0)
    got = F.cpu().numpy()
    assert got.shape == (nx, ny)
    assert np.all(np.abs(got - ref) <= 1e-13 * np.abs(v).sum(axis=0) * (wa[-1] - wa[0]) * 1e-8)
    with pytest.raises(OcoError):  # plane of another grid size
        e.integrated_flux_device(vt[:10], (nx, ny))
    e.set_wavelengths(wa[:1])
    one = e.integrated_flux_device(vt[:1].contiguous(), (nx, ny))
    e.synchronize()
    assert np.array_equal(one.cpu().numpy(), np.zeros((nx, ny)))
    e.close()
