"""The solve entry point that allocates no GPU memory, through the C ABI.

Some callers cannot call cudaMalloc (hosts that own the device heap, plugins that may not
allocate after start-up, drivers with a fixed GPU-memory budget).  oco_solve_block_noalloc
serves them from a static device workspace compiled into the library.  Here it must give the
same bits as the regular device entry point, on several calls in a row with different problems
(the shared workspace keeps the previous call's contents, so each later call also checks that
everything is re-initialised):
  - a generic-path plain case and a stable case (nw < 64, one chunk each);
  - a staged-path case (nw = 64) whose columns need several chunks of the workspace;
  - the documented size limit nz = OCO_NOALLOC_MAX_NZ with nw = OCO_NOALLOC_MAX_NW;
  - a call with U omitted (NULL), as the regular entry point allows.
This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_NZ = 4096  # OCO_NOALLOC_MAX_NZ in include/oco.h
MAX_NW = 4096  # OCO_NOALLOC_MAX_NW


def _bitwise(a, b, what):
    na, nb = np.isnan(a), np.isnan(b)
    assert np.array_equal(na, nb), what
    assert np.array_equal(a[~na].view(np.uint64), b[~nb].view(np.uint64)), what


def _compare(lib, eng, dev, nx, ny, nz, nw, form, layout, seed, wa=None, keep=("U", "kappa", "V", "Vtop", "Vbot")):
    import torch
    from ocotillo_b200 import workloads
    from ocotillo_b200.engine import _DP

    rho_h, T_h, dz = workloads.agn_block(nx, ny, nz, seed=seed)
    wa = workloads.log_wavelengths(nw) if wa is None else wa
    rho = torch.from_numpy(rho_h).to(dev)
    T = torch.from_numpy(T_h).to(dev)
    if layout == 0:
        shp = {"U": (nw, nx, ny, nz + 6), "kappa": (nw, nx, ny, nz), "V": (nw, nx, ny, nz)}
    else:
        shp = {"U": (nz + 6, nx * ny, nw), "kappa": (nz, nx * ny, nw), "V": (nz, nx * ny, nw)}
    shp["Vtop"] = shp["Vbot"] = (nw, nx, ny)
    shp = {k: v for k, v in shp.items() if k in keep}

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
    ptr = lambda k: ctypes.c_void_p(got[k].data_ptr()) if k in got else None
    rc = lib.oco_solve_block_noalloc(ctypes.byref(prm), wa_c.ctypes.data_as(_DP), ctypes.c_void_p(rho.data_ptr()),
                                     ctypes.c_void_p(T.data_ptr()), ptr("U"), ptr("kappa"), ptr("V"), ptr("Vtop"),
                                     ptr("Vbot"), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == ref_rc, lib.oco_noalloc_last_error()
    for k in shp:
        _bitwise(got[k].cpu().numpy(), ref[k].cpu().numpy(), f"{form} layout {layout} nz {nz} nw {nw} {k}")


def test_noalloc_matches_regular_entry_point_on_calls_in_a_row():
    import torch
    from ocotillo_b200 import Engine
    from ocotillo_b200.engine import load_library

    lib = load_library()
    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    eng = Engine(0)
    _compare(lib, eng, dev, 4, 6, 64, 40, "plain", 0, 21)
    _compare(lib, eng, dev, 5, 3, 33, 17, "stable", 1, 22)
    # staged path (nw = 64) with 128 columns of nz = 1024: the workspace holds ~74 columns of
    # pillar records beside its scratch, so the call runs two chunks (second one at c_off > 0)
    _compare(lib, eng, dev, 8, 16, 1024, 64, "plain", 0, 23)
    # U omitted
    _compare(lib, eng, dev, 2, 3, 40, 64, "stable", 1, 24, keep=("kappa", "V", "Vtop", "Vbot"))
    eng.close()


def test_noalloc_accepts_the_documented_limits():
    """nz = OCO_NOALLOC_MAX_NZ with the largest wavelength grid: one 128-thread block of scratch
    and one column of records beside the largest table."""
    import torch
    from ocotillo_b200 import Engine, workloads
    from ocotillo_b200.engine import load_library

    lib = load_library()
    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    eng = Engine(0)
    _compare(lib, eng, dev, 1, 1, MAX_NZ, MAX_NW, "stable", 1, 25, wa=workloads.log_wavelengths(MAX_NW),
             keep=("kappa", "Vtop", "Vbot"))
    eng.close()


def test_noalloc_rejects_sizes_beyond_the_workspace():
    import torch
    from ocotillo_b200.engine import load_library, OcoParams, _DP

    lib = load_library()
    torch.cuda.set_device(0)
    for nz, nw in ((MAX_NZ + 1, 8), (64, MAX_NW + 1)):
        prm = OcoParams(1, 1, nz, nw, 1e13, 0.4, 2e4, 0, 0, 0, 0)
        wa = np.linspace(1000.0, 2000.0, nw)
        rc = lib.oco_solve_block_noalloc(ctypes.byref(prm), wa.ctypes.data_as(_DP), ctypes.c_void_p(1),
                                         ctypes.c_void_p(1), ctypes.c_void_p(1), None, None, None, None, None)
        assert rc == -1
        assert b"exceed" in lib.oco_noalloc_last_error()
