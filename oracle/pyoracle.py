"""ctypes wrapper of the C oracle (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this module.
The oracle restates the reference's xy/lambda loop (flux_feautrier.f90:160-228) on the CPU;
see oco_oracle.h.  Arrays use the reference's Fortran layouts:
  rho, T : (nx, ny, nz) C-order == Fortran (nz, ny, nx)
  U      : (nw, nx, ny, nz+6), kappa and V : (nw, nx, ny, nz)
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")

FORM_REFERENCE = 0
FORM_STABLE = 1


class OracleParams(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32), ("nw", ctypes.c_int32),
        ("dz", ctypes.c_double), ("lgrey", ctypes.c_int32), ("form", ctypes.c_int32),
        ("sigma_grey", ctypes.c_double), ("fully_ionized_T", ctypes.c_double),
    ]


def build():
    """Compile the oracle libraries (gcc, make)."""
    subprocess.check_call(["make", "-s", "-C", HERE], stdout=subprocess.DEVNULL)


_LIBS = {}


def _lib(backend):
    if backend not in _LIBS:
        path = os.path.join(BUILD, f"liboco_oracle_{backend}.so")
        if not os.path.exists(path):
            build()
        lib = ctypes.CDLL(path)
        P = ctypes.POINTER(ctypes.c_double)
        lib.oracle_solve_columns.argtypes = [ctypes.POINTER(OracleParams), P, P, P, ctypes.c_int64,
                                             ctypes.c_int64, P, P, P, ctypes.POINTER(ctypes.c_int64)]
        lib.oracle_solve_columns.restype = ctypes.c_int
        lib.oracle_run_deck.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int]
        lib.oracle_run_deck.restype = ctypes.c_int
        lib.oracle_format_e.argtypes = [ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_char_p]
        lib.oracle_calc_wavelength.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_int32, P]
        lib.oracle_math_backend.restype = ctypes.c_int
        _LIBS[backend] = lib
    return _LIBS[backend]


def _ptr(a):
    if a is None:
        return None
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def solve_block(rho, T, wa, dz, fully_ionized_T=2e4, lgrey=False, sigma_grey=0.4,
                form=FORM_REFERENCE, backend="ocomath", want=("U", "kappa", "V")):
    """Runs the oracle on a block.  rho, T: float64 arrays of shape (nx, ny, nz)."""
    rho = np.ascontiguousarray(rho, dtype=np.float64)
    T = np.ascontiguousarray(T, dtype=np.float64)
    wa = np.ascontiguousarray(np.atleast_1d(wa), dtype=np.float64)
    nx, ny, nz = rho.shape
    nw = wa.shape[0]
    prm = OracleParams(nx, ny, nz, nw, float(dz), int(bool(lgrey)), int(form), float(sigma_grey),
                       float(fully_ionized_T))
    U = np.empty((nw, nx, ny, nz + 6)) if "U" in want else None
    K = np.empty((nw, nx, ny, nz)) if "kappa" in want else None
    V = np.empty((nw, nx, ny, nz)) if "V" in want else None
    bad = ctypes.c_int64(-1)
    rc = _lib(backend).oracle_solve_columns(ctypes.byref(prm), _ptr(wa), _ptr(rho), _ptr(T), 0, nx * ny,
                                            _ptr(U), _ptr(K), _ptr(V), ctypes.byref(bad))
    return {"rc": rc, "bad_item": bad.value, "U": U, "kappa": K, "V": V}


def run_deck(deck_dir, out_dir, backend="glibc"):
    msg = ctypes.create_string_buffer(512)
    rc = _lib(backend).oracle_run_deck(deck_dir.encode(), out_dir.encode(), msg, 512)
    return rc, msg.value.decode()


def format_e(v, w=15, d=5):
    buf = ctypes.create_string_buffer(w + 1)
    _lib("glibc").oracle_format_e(float(v), w, d, buf)
    return buf.value.decode()


def calc_wavelength(w1, w0, nw):
    wa = np.empty(nw)
    _lib("glibc").oracle_calc_wavelength(float(w1), float(w0), nw, _ptr(wa))
    return wa


_MC = None


def mathcheck(kind, fn, x, y=None):
    """Element-wise reference math: kind in {'glibc', 'quad', 'ocomath'};
    fn in {'exp', 'log', 'log10', 'pow', 'pow10'} ('pow10': ocomath only)."""
    global _MC
    if _MC is None:
        path = os.path.join(BUILD, "libmathcheck.so")
        if not os.path.exists(path):
            build()
        _MC = ctypes.CDLL(path)
        for name in ("mc_glibc", "mc_quad", "mc_ocomath"):
            f = getattr(_MC, name)
            f.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                          ctypes.POINTER(ctypes.c_double), ctypes.c_int64]
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y if y is not None else np.zeros_like(x), dtype=np.float64)
    out = np.empty_like(x)
    code = {"exp": 0, "log": 1, "log10": 2, "pow": 3, "pow10": 4}[fn]
    getattr(_MC, "mc_" + kind)(code, _ptr(x), _ptr(y), _ptr(out), x.size)
    return out
