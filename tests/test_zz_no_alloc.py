"""The solve entry point that allocates no GPU memory, through the C ABI.

Some callers cannot call cudaMalloc (hosts that own the device heap, plugins that may not
allocate after start-up, drivers with a fixed GPU-memory budget).  oco_solve_block_noalloc
serves them from a static device workspace compiled into the library.  Here it must give the
same bits as the regular device entry point, on two calls in a row with different problems
(the shared workspace keeps the previous call's contents, so the second call also checks
that everything is re-initialised).  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bitwise(a, b, what):
    na, nb = np.isnan(a), np.isnan(b)
    assert np.array_equal(na, nb), what
    assert np.array_equal(a[~na].view(np.uint64), b[~nb].view(np.uint64)), what


def test_noalloc_matches_regular_entry_point_twice():
    import torch
    from ocotillo_b200 import Engine, workloads
    from ocotillo_b200.engine import load_library, _DP

    lib = load_library()
    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    eng = Engine(0)
    cases = [(4, 6, 64, 40, "plain", 0, 21), (5, 3, 33, 17, "stable", 1, 22)]
    for nx, ny, nz, nw, form, layout, seed in cases:
        rho_h, T_h, dz = workloads.agn_block(nx, ny, nz, seed=seed)
        wa = workloads.log_wavelengths(nw)
        rho = torch.from_numpy(rho_h).to(dev)
        T = torch.from_numpy(T_h).to(dev)
        if layout == 0:
            shp = {"U": (nw, nx, ny, nz + 6), "kappa": (nw, nx, ny, nz), "V": (nw, nx, ny, nz)}
        else:
            shp = {"U": (nz + 6, nx * ny, nw), "kappa": (nz, nx * ny, nw), "V": (nz, nx * ny, nw)}
        shp["Vtop"] = shp["Vbot"] = (nw, nx, ny)

        def fresh():
            return {k: torch.full(s, float("nan"), dtype=torch.float64, device=dev) for k, s in shp.items()}

        ref = fresh()
        eng.set_wavelengths(wa)
        eng.solve_block_device(rho, T, dz, ref, form=form, layout=layout)
        torch.cuda.synchronize()
        try:
            eng.synchronize()
            ref_rc = 0
        except Exception as e:
            ref_rc = e.code
        got = fresh()
        prm = eng.params(rho_h.shape, nw, dz, form=form, layout=layout)
        wa_c = np.ascontiguousarray(wa)
        ptr = lambda t: ctypes.c_void_p(t.data_ptr())
        rc = lib.oco_solve_block_noalloc(ctypes.byref(prm), wa_c.ctypes.data_as(_DP), ptr(rho), ptr(T),
                                         ptr(got["U"]), ptr(got["kappa"]), ptr(got["V"]), ptr(got["Vtop"]),
                                         ptr(got["Vbot"]), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
        assert rc == ref_rc, lib.oco_noalloc_last_error()
        for k in shp:
            _bitwise(got[k].cpu().numpy(), ref[k].cpu().numpy(), f"{form} layout {layout} {k}")
    eng.close()


def test_noalloc_rejects_sizes_beyond_the_workspace():
    import torch
    from ocotillo_b200 import Engine
    from ocotillo_b200.engine import load_library, OcoParams, _DP

    lib = load_library()
    torch.cuda.set_device(0)
    prm = OcoParams(1, 1, 5000, 8, 1e13, 0.4, 2e4, 0, 0, 0, 0)
    wa = np.linspace(1000.0, 2000.0, 8)
    rc = lib.oco_solve_block_noalloc(ctypes.byref(prm), wa.ctypes.data_as(_DP), ctypes.c_void_p(1),
                                     ctypes.c_void_p(1), ctypes.c_void_p(1), None, None, None, None, None)
    assert rc == -1
    assert b"exceed" in lib.oco_noalloc_last_error()
