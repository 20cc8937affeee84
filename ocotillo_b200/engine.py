"""ctypes binding of include/oco.h.

Mirrors the reference's interface for the hot path: calc_wavelength
(continuous_opacity.f90:37-62), pre_calc_opacity_quantities (:64-141, here
Engine.set_wavelengths) and the xy/lambda loop of flux_feautrier.f90:160-228
(Engine.solve_block for host arrays, Engine.solve_block_device for torch CUDA tensors).
Array shapes follow the reference's Fortran arrays read in C order:
  rho, T       (nx, ny, nz)          == Fortran (nz, ny, nx)
  U            (nw, nx, ny, nz+6)    == Fortran U(mz, ny, nx, nw)
  kappa, V     (nw, nx, ny, nz)
  Vtop, Vbot   (nw, nx, ny)          V at z index nz and 1
The device entry point also offers the lambda-fastest layout:
  U (nz+6, nx*ny, nw), kappa and V (nz, nx*ny, nw).
"""
import ctypes
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "liboco_b200.so")

FORM_PLAIN, FORM_STABLE, FORM_MIXED = 0, 1, 2
LAYOUT_REFERENCE, LAYOUT_LAMBDA_FASTEST = 0, 1
_FORMS = {"plain": FORM_PLAIN, "stable": FORM_STABLE, "mixed": FORM_MIXED}

OCO_OK = 0
ERRORS = {-1: "EINVAL", -2: "ENOMEM", -3: "EZEROPIVOT", -4: "EGREY", -5: "ECUDA", -6: "ETIMEDOUT",
          -7: "EAGAIN", -8: "EADMIT", -9: "EIO", -10: "EDIM", -11: "ENOWAVES", -12: "ENAN", -13: "ECLOSED"}


class OcoError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class OcoParams(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32), ("nw", ctypes.c_int32),
                ("dz", ctypes.c_double), ("sigma_grey", ctypes.c_double), ("fully_ionized_T", ctypes.c_double),
                ("lgrey", ctypes.c_int32), ("form", ctypes.c_int32), ("layout", ctypes.c_int32),
                ("reserved", ctypes.c_int32)]


_LIB = None
_DP = ctypes.POINTER(ctypes.c_double)


def load_library(path=None):
    """Loads liboco_b200.so (built in-tree by ocotillo_b200.build).  Raises if absent."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = path or LIB_PATH
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with `python -m ocotillo_b200.build`")
    lib = ctypes.CDLL(path)
    V, I, P, D = ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(OcoParams), ctypes.c_double
    sig = {
        "oco_abi_version": (I, []),
        "oco_create": (I, [ctypes.POINTER(V), I]),
        "oco_destroy": (None, [V]),
        "oco_last_error": (ctypes.c_char_p, [V]),
        "oco_calc_wavelength": (I, [D, D, ctypes.c_int32, _DP]),
        "oco_set_wavelengths": (I, [V, _DP, ctypes.c_int32]),
        "oco_solve_block": (I, [V, P, _DP, _DP, _DP, _DP, _DP, _DP, _DP]),
        "oco_solve_block_device": (I, [V, P, V, V, V, V, V, V, V, V]),
        "oco_synchronize": (I, [V]),
        "oco_kernel_launches": (ctypes.c_int64, [V]),
        "oco_set_profiling": (I, [V, I]),
        "oco_kernel_times": (I, [V, _DP, _DP, ctypes.POINTER(ctypes.c_int64)]),
        "oco_solve_block_noalloc": (I, [P, _DP, V, V, V, V, V, V, V, V]),
        "oco_noalloc_last_error": (ctypes.c_char_p, []),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _LIB = lib
    return lib


def _ptr(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_DP)


def calc_wavelength(w1, w0, nw):
    """Linear grid of continuous_opacity.f90:37-62 (argument order as there)."""
    lib = load_library()
    wa = np.empty(nw)
    rc = lib.oco_calc_wavelength(float(w1), float(w0), int(nw), _ptr(wa))
    if rc:
        raise OcoError(rc, lib.oco_last_error(None).decode())
    return wa


class Engine:
    """One context of the engine on one CUDA device."""

    def __init__(self, device=0):
        self.lib = load_library()
        self.ctx = ctypes.c_void_p()
        rc = self.lib.oco_create(ctypes.byref(self.ctx), int(device))
        if rc:
            raise OcoError(rc, self.lib.oco_last_error(None).decode())
        self.device = device
        self.nw = 0

    def close(self):
        if self.ctx:
            self.lib.oco_destroy(self.ctx)
            self.ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc:
            raise OcoError(rc, self.lib.oco_last_error(self.ctx).decode())

    def set_wavelengths(self, wa):
        """pre_calc_opacity_quantities for a wavelength grid in Angstrom."""
        wa = np.ascontiguousarray(np.atleast_1d(wa), dtype=np.float64)
        self._check(self.lib.oco_set_wavelengths(self.ctx, _ptr(wa), wa.size))
        self.nw = wa.size

    def params(self, shape, nw, dz, fully_ionized_T=2e4, lgrey=False, sigma_grey=0.4, form="plain",
               layout=LAYOUT_REFERENCE):
        nx, ny, nz = shape
        return OcoParams(nx, ny, nz, nw, float(dz), float(sigma_grey), float(fully_ionized_T), int(bool(lgrey)),
                         _FORMS[form] if isinstance(form, str) else int(form), int(layout), 0)

    def solve_block(self, rho, T, dz, fully_ionized_T=2e4, lgrey=False, sigma_grey=0.4, form="plain",
                    want=("U", "kappa", "V", "Vtop", "Vbot"), out=None, allow_zero_pivot=False):
        """The reference's xy/lambda loop on host arrays.  rho, T: (nx, ny, nz) float64.
        Returns a dict of numpy arrays (reference layout).  `out` may supply preallocated
        (e.g. pinned) arrays by name.  An exactly zero Thomas pivot raises OcoError
        (EZEROPIVOT), as the reference stops there; with allow_zero_pivot=True the results
        are returned with out['zero_pivot'] = True instead."""
        rho = np.ascontiguousarray(rho, dtype=np.float64)
        T = np.ascontiguousarray(T, dtype=np.float64)
        nx, ny, nz = rho.shape
        nw = 1 if lgrey else self.nw
        out = dict(out or {})
        shapes = {"U": (nw, nx, ny, nz + 6), "kappa": (nw, nx, ny, nz), "V": (nw, nx, ny, nz),
                  "Vtop": (nw, nx, ny), "Vbot": (nw, nx, ny)}
        for k in set(want) | {"U"}:
            if k not in out:
                out[k] = np.empty(shapes[k])
        prm = self.params(rho.shape, nw, dz, fully_ionized_T, lgrey, sigma_grey, form)
        rc = self.lib.oco_solve_block(self.ctx, ctypes.byref(prm), _ptr(rho), _ptr(T), _ptr(out.get("U")),
                                      _ptr(out.get("kappa")), _ptr(out.get("V")), _ptr(out.get("Vtop")),
                                      _ptr(out.get("Vbot")))
        out["zero_pivot"] = rc == -3
        if not (rc == -3 and allow_zero_pivot):
            self._check(rc)
        return out

    def solve_block_device(self, rho, T, dz, out, fully_ionized_T=2e4, lgrey=False, sigma_grey=0.4,
                           form="plain", layout=LAYOUT_REFERENCE, stream=None):
        """Same loop on torch CUDA tensors (float64, contiguous), enqueued on `stream`
        (default: torch's current stream).  `out` maps 'U' (required), 'kappa', 'V', 'Vtop',
        'Vbot' to preallocated tensors of the layout's shapes."""
        import torch
        nx, ny, nz = rho.shape
        nw = 1 if lgrey else self.nw
        for t in [rho, T] + [v for v in out.values() if v is not None]:
            assert t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()
        if stream is None:
            stream = torch.cuda.current_stream(rho.device)
        prm = self.params(rho.shape, nw, dz, fully_ionized_T, lgrey, sigma_grey, form, layout)

        def p(name):
            t = out.get(name)
            return ctypes.c_void_p(t.data_ptr()) if t is not None else None

        rc = self.lib.oco_solve_block_device(self.ctx, ctypes.byref(prm), ctypes.c_void_p(rho.data_ptr()),
                                             ctypes.c_void_p(T.data_ptr()), p("U"), p("kappa"), p("V"),
                                             p("Vtop"), p("Vbot"), ctypes.c_void_p(stream.cuda_stream))
        self._check(rc)
        return out

    def synchronize(self):
        self._check(self.lib.oco_synchronize(self.ctx))

    @property
    def kernel_launches(self):
        return self.lib.oco_kernel_launches(self.ctx)

    def set_profiling(self, enable=True):
        self._check(self.lib.oco_set_profiling(self.ctx, int(bool(enable))))

    def kernel_times(self):
        """(solve_ms, pillars_ms, solve_launches) since the last call (profiling on)."""
        a, b, n = ctypes.c_double(), ctypes.c_double(), ctypes.c_int64()
        self._check(self.lib.oco_kernel_times(self.ctx, ctypes.byref(a), ctypes.byref(b), ctypes.byref(n)))
        return a.value, b.value, n.value
