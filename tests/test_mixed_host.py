"""The mixed form's arithmetic (mixed_core.h) compiled for the host, against the stable FP64
oracle at the mixed form's tolerances: kappa 3e-5, U 5e-4, emergent flux 1e-4 (relative).  The
GPU kernels inline the same functions (with the SFU's ex2/lg2 for libm's exp2f/log2f), so this
catches a regression in the arithmetic without a GPU."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "ocotillo_b200")
BUILD = os.path.join(ROOT, "tests", "_build")
P = ctypes.POINTER(ctypes.c_double)


@pytest.fixture(scope="module")
def host_lib():
    lib = os.path.join(PKG, "liboco_b200.so")
    if not os.path.exists(lib):
        pytest.fail("liboco_b200.so is missing: build it with `python -m ocotillo_b200.build`")
    os.makedirs(BUILD, exist_ok=True)
    out = os.path.join(BUILD, "libmixed_host.so")
    src = os.path.join(ROOT, "tests", "mixed_host.cpp")
    cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off", "-I", os.path.join(PKG, "csrc"),
           "-I", "/usr/local/cuda/include", "-o", out, src, f"-L{PKG}", "-l:liboco_b200.so", f"-Wl,-rpath,{PKG}"]
    subprocess.run(cmd, check=True, capture_output=True)
    h = ctypes.CDLL(out)
    h.mixed_host_solve.argtypes = [P, P, P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                   ctypes.c_double, P, P, P]
    return h


def _solve(h, rho, T, wa, dz):
    ncol, nz = rho.shape
    nw = len(wa)
    U = np.zeros(nw * ncol * (nz + 6))
    K = np.zeros(nw * ncol * nz)
    V = np.zeros(nw * ncol * nz)
    p = lambda a: a.ctypes.data_as(P)
    h.mixed_host_solve(p(np.ascontiguousarray(rho)), p(np.ascontiguousarray(T)), p(wa), ncol, nz, nw, dz, 2e4,
                       p(U), p(K), p(V))
    return U.reshape(nw, ncol, nz + 6), K.reshape(nw, ncol, nz), V.reshape(nw, ncol, nz)


@pytest.mark.parametrize("case", ["agn", "athena"])
def test_mixed_host_against_stable_oracle(host_lib, oracle, case):
    from ocotillo_b200 import workloads
    if case == "agn":
        rho, T, dz = workloads.agn_block(2, 3, 160, seed=31)
        wa = workloads.log_wavelengths(48)
    else:
        rng = np.random.default_rng(32)
        cols = [workloads.athena_column(120, rng, sigma_dex=0.3) for _ in range(4)]
        rho = np.stack([c[0] for c in cols]).reshape(4, 1, 120)
        T = np.stack([c[1] for c in cols]).reshape(4, 1, 120)
        dz = cols[0][2]
        wa = workloads.log_wavelengths(40, 900.0, 40000.0)
    nx, ny, nz = rho.shape
    U, K, V = _solve(host_lib, rho.reshape(-1, nz), T.reshape(-1, nz), wa, dz)
    ref = oracle.solve_block(rho, T, wa, dz, form=oracle.FORM_STABLE, backend="ocomath")
    nw = len(wa)
    rU = ref["U"].reshape(nw, nx * ny, nz + 6)
    rK = ref["kappa"].reshape(nw, nx * ny, nz)
    rV = ref["V"].reshape(nw, nx * ny, nz)
    rel = lambda a, b: np.abs(a - b) / np.maximum(np.abs(b), 1e-300)
    assert rel(K, rK).max() <= 3e-5
    assert rel(U, rU).max() <= 5e-4
    for end in (-1, 0):
        assert rel(V[..., end], rV[..., end]).max() <= 1e-4, end


@pytest.mark.parametrize("rho0", [1e-11, 1e-9, 1e-7])
def test_mixed_host_across_precision_config_densities(host_lib, oracle, rho0):
    """The precision workload draws rho0 log-uniform in [1e-11, 1e-7]: its ends and middle, at the
    mixed form's tolerances against the stable FP64 oracle."""
    from ocotillo_b200 import workloads
    rho, T, dz = workloads.agn_block(2, 2, 160, seed=41, rho0=rho0)
    wa = workloads.log_wavelengths(48)
    nx, ny, nz = rho.shape
    nw = len(wa)
    U, K, V = _solve(host_lib, rho.reshape(-1, nz), T.reshape(-1, nz), wa, dz)
    ref = oracle.solve_block(rho, T, wa, dz, form=oracle.FORM_STABLE, backend="ocomath")
    rel = lambda a, b: np.abs(a - b) / np.maximum(np.abs(b), 1e-300)
    assert rel(K, ref["kappa"].reshape(nw, nx * ny, nz)).max() <= 3e-5
    assert rel(U, ref["U"].reshape(nw, nx * ny, nz + 6)).max() <= 5e-4
    rV = ref["V"].reshape(nw, nx * ny, nz)
    for end in (-1, 0):
        assert rel(V[..., end], rV[..., end]).max() <= 1e-4, end


@pytest.mark.parametrize("nz,nw", [(2, 7), (3, 40), (4, 33), (5, 64), (9, 31)])
def test_mixed_host_short_columns(host_lib, oracle, nz, nw):
    """Short columns (the ghost zones of nz < 4 feed each other).  For nz < 4 the reference's
    stencil on U differences values below FP64 resolution in these optically thin columns, so
    the flux is rounding noise in any precision and only kappa and U are compared."""
    from ocotillo_b200 import workloads
    rho, T, _ = workloads.agn_block(2, 3, nz, seed=nz + 40)
    dz = 2.5e14
    wa = workloads.log_wavelengths(nw, 1000.0, 30000.0)
    U, K, V = _solve(host_lib, rho.reshape(-1, nz), T.reshape(-1, nz), wa, dz)
    ref = oracle.solve_block(rho, T, wa, dz, form=oracle.FORM_STABLE, backend="ocomath")
    rel = lambda a, b: np.abs(a - b) / np.maximum(np.abs(b), 1e-300)
    assert np.isfinite(U).all() and np.isfinite(V).all()
    assert rel(K, ref["kappa"].reshape(nw, 6, nz)).max() <= 3e-5
    assert rel(U, ref["U"].reshape(nw, 6, nz + 6)).max() <= 5e-4
    if nz >= 4:
        rV = ref["V"].reshape(nw, 6, nz)
        for end in (-1, 0):
            assert rel(V[..., end], rV[..., end]).max() <= 1e-4, end


def test_scratch_record_packing(host_lib):
    """The ragged-batch kernels' 12-byte scratch record packs u's exponent into the spare bits
    of 1/kappa (> 0) and of u's mantissa (in [1, 2)): every fitting record comes back with the
    same bits, and every record outside the packable range reports that it does not fit (the
    kernel then flags the item for the FP64 re-solve)."""
    rng = np.random.default_rng(7)
    n = 200000
    o1 = (10.0 ** rng.uniform(-38, 38, n)).astype(np.float32)
    m = (1.0 + rng.random(n)).astype(np.float32)
    m[m >= 2.0] = np.float32(1.9999999)
    e = rng.integers(-600, 600, n).astype(np.int32)
    edge = np.array([-512, 511, -513, 512, 0, -1], dtype=np.int32)
    e[:edge.size] = edge
    o1[:4] = [np.float32(1.0), np.finfo(np.float32).max, np.finfo(np.float32).tiny, np.float32(3e-39)]
    m[6:12] = [1.0, np.nextafter(np.float32(2.0), np.float32(0.0)), 0.0, 2.0, 0.5, -1.5]
    fits = np.zeros(n, dtype=np.int32)
    o1r = np.zeros(n, dtype=np.float32)
    mr = np.zeros(n, dtype=np.float32)
    er = np.zeros(n, dtype=np.int32)
    pf = ctypes.POINTER(ctypes.c_float)
    pi = ctypes.POINTER(ctypes.c_int)
    host_lib.mixed_host_pack_roundtrip.argtypes = [pf, pf, pi, ctypes.c_int, pi, pf, pf, pi]
    host_lib.mixed_host_pack_roundtrip(o1.ctypes.data_as(pf), m.ctypes.data_as(pf), e.ctypes.data_as(pi), n,
                                       fits.ctypes.data_as(pi), o1r.ctypes.data_as(pf), mr.ctypes.data_as(pf),
                                       er.ctypes.data_as(pi))
    normal_m = (m >= 1.0) & (m < 2.0)
    expect = (e >= -512) & (e <= 511) & normal_m
    assert np.array_equal(fits.astype(bool), expect)
    ok = expect
    assert ok.sum() > n // 2
    assert np.array_equal(o1r[ok].view(np.uint32), o1[ok].view(np.uint32))
    assert np.array_equal(mr[ok].view(np.uint32), m[ok].view(np.uint32))
    assert np.array_equal(er[ok], e[ok])


@pytest.mark.parametrize("case", ["agn", "precision", "athena"])
def test_u_exponents_fit_the_packed_scratch_record(host_lib, case):
    """The ragged-batch kernels pack u's binary exponent into 10 bits (e + 512 in [0, 1023]) and
    rely on u's mantissa lying in [1, 2); an item whose records do not fit is flagged for the
    FP64 re-solve, so this is about cost, not correctness.  On the benchmark constructions the
    forward sweep's u keeps its mantissa normalised and its exponent well inside the range."""
    from ocotillo_b200 import workloads
    if case == "agn":
        rho, T, dz = workloads.agn_block(2, 2, 512)
        wa = workloads.log_wavelengths(64)
    elif case == "precision":
        rho, T, dz, _ = workloads.precision_block(2, 1, 1024)
        wa = workloads.log_wavelengths(64)
    else:
        rng = np.random.default_rng(4)
        cols = [workloads.athena_column(nz, rng) for nz in (64, 300, 2048)]
        out = []
        for r, t, d in cols:
            out.append(_exponents(host_lib, r.reshape(1, -1), t.reshape(1, -1), workloads.log_wavelengths(48), d))
        emin, emax, bad = min(o[0] for o in out), max(o[1] for o in out), sum(o[2] for o in out)
        assert bad == 0 and -480 <= emin and emax <= 400, (emin, emax, bad)
        return
    nz = rho.shape[-1]
    emin, emax, bad = _exponents(host_lib, rho.reshape(-1, nz), T.reshape(-1, nz), wa, dz)
    assert bad == 0 and -480 <= emin and emax <= 400, (emin, emax, bad)


def _exponents(h, rho, T, wa, dz):
    ncol, nz = rho.shape
    out = (ctypes.c_int * 3)()
    h.mixed_host_u_exponents.argtypes = [P, P, P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                         ctypes.c_double, ctypes.POINTER(ctypes.c_int)]
    p = lambda a: np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(P)
    wa = np.ascontiguousarray(wa, dtype=np.float64)
    h.mixed_host_u_exponents(p(rho), p(T), wa.ctypes.data_as(P), ncol, nz, len(wa), dz, 2e4, out)
    return out[0], out[1], out[2]
