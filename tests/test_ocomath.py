"""The shared math core (ocomath) on the host: accuracy and special cases.

ocomath is what both the GPU kernels and the oracle's 'ocomath' back-end call, so the GPU and
CPU agree bit for bit.  Here it is checked against quad-precision references rounded to
double (correct rounding except within 2^-113 of a boundary) and against glibc, which the
gfortran-built reference calls.  The glibc mismatch rate is the 'libm floor' between any
faithful re-implementation and the reference binary.
"""
import numpy as np
import pytest

N = 200_000


def _inputs(fn, rng):
    if fn == "exp":
        return rng.uniform(-745.2, 709.78, N), None
    if fn in ("log", "log10"):
        return np.exp(rng.uniform(-700, 700, N)), None
    return np.exp(rng.uniform(-10, 10, N)), rng.uniform(-20, 20, N)


@pytest.mark.parametrize("fn", ["exp", "log", "log10", "pow"])
def test_correctly_rounded_vs_quad(oracle, fn):
    rng = np.random.default_rng(11)
    x, y = _inputs(fn, rng)
    a = oracle.mathcheck("ocomath", fn, x, y)
    q = oracle.mathcheck("quad", fn, x, y)
    assert np.array_equal(a, q), f"{fn}: {np.count_nonzero(a != q)} of {N} differ from the quad reference"


def test_pow10_correctly_rounded(oracle):
    rng = np.random.default_rng(12)
    t = rng.uniform(-320, 308, N)
    x = np.full(N, 10.0)
    assert np.array_equal(oracle.mathcheck("ocomath", "pow", x, t), oracle.mathcheck("quad", "pow", x, t))


def test_subnormal_exp_range(oracle):
    rng = np.random.default_rng(13)
    x = rng.uniform(-745.2, -708.0, N)
    assert np.array_equal(oracle.mathcheck("ocomath", "exp", x), oracle.mathcheck("quad", "exp", x))


@pytest.mark.parametrize("fn,limit", [("exp", 5e-3), ("log", 1e-4), ("pow", 5e-3), ("log10", 1e-2)])
def test_libm_floor_vs_glibc(oracle, fn, limit):
    # Not an error bound of ocomath: the fraction of calls where glibc itself is not
    # correctly rounded.  Recorded so that a regression in either is visible.
    rng = np.random.default_rng(14)
    x, y = _inputs(fn, rng)
    a = oracle.mathcheck("ocomath", fn, x, y)
    g = oracle.mathcheck("glibc", fn, x, y)
    frac = np.count_nonzero(a != g) / N
    assert frac < limit


SPECIAL_POW = [(0.0, 1.0), (0.0, -1.0), (-0.0, -3.0), (-0.0, 3.0), (-2.0, 3.0), (-2.0, 0.5),
               (1.0, np.nan), (np.nan, 0.0), (np.inf, -1.0), (-np.inf, 3.0), (-np.inf, 2.0),
               (0.5, np.inf), (2.0, -np.inf), (-1.0, np.inf), (1e-310, 0.5), (5e-324, 1.0),
               (2.0, 1023.9), (2.0, 1024.0), (2.0, -1074.0), (2.0, -1075.0), (10.0, 308.3),
               (10.0, -323.5), (-8.0, 1.0 / 3.0), (np.nan, 1.0), (3.0, np.nan)]


def test_pow_special_cases_match_glibc(oracle):
    x = np.array([a for a, _ in SPECIAL_POW])
    y = np.array([b for _, b in SPECIAL_POW])
    a = oracle.mathcheck("ocomath", "pow", x, y)
    g = oracle.mathcheck("glibc", "pow", x, y)
    same = (a == g) | (np.isnan(a) & np.isnan(g))
    assert same.all(), list(zip(x[~same], y[~same], a[~same], g[~same]))
    fin = ~np.isnan(a)
    assert np.array_equal(np.signbit(a[fin]), np.signbit(g[fin]))


def test_exp_log_special_cases(oracle):
    x = np.array([-746.5, -745.2, -745.1332191019412, -745.13, -708.4, 709.78, 709.79, 0.0, -0.0,
                  1e-300, np.inf, -np.inf, np.nan])
    a, g = oracle.mathcheck("ocomath", "exp", x), oracle.mathcheck("glibc", "exp", x)
    assert (((a == g) | (np.isnan(a) & np.isnan(g)))).all()
    x = np.array([1.0, 5e-324, 2.2250738585072014e-308, 1e-310, 1.7976931348623157e308, 0.75, 1.5,
                  10.0, 100.0, 0.0, -1.0, np.inf, np.nan])
    for fn in ("log", "log10"):
        a, q = oracle.mathcheck("ocomath", fn, x), oracle.mathcheck("quad", fn, x)
        assert (((a == q) | (np.isnan(a) & np.isnan(q)))).all(), fn
    assert oracle.mathcheck("ocomath", "log", np.array([1.0]))[0] == 0.0


def test_pow10_fast_path_is_pow_of_ten(oracle):
    # The kernels call oco_pow10(y); the oracle calls oco_pow(10.0, y).  They must agree
    # bit for bit everywhere, including the special values.
    rng = np.random.default_rng(15)
    y = np.concatenate([rng.uniform(-330, 310, N), [0.0, -0.0, np.inf, -np.inf, 1e-300, -1e-300, 308.2547,
                                                    308.26, -323.3, -324.5, 400.0, -400.0]])
    a = oracle.mathcheck("ocomath", "pow10", y, y)
    b = oracle.mathcheck("ocomath", "pow", np.full_like(y, 10.0), y)
    assert np.array_equal(a.view(np.uint64), b.view(np.uint64))
    nan = oracle.mathcheck("ocomath", "pow10", np.array([np.nan]), np.array([np.nan]))
    assert np.isnan(nan).all()


@pytest.fixture(scope="module")
def exp_host():
    import ctypes
    import os
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    build = os.path.join(root, "tests", "_build")
    os.makedirs(build, exist_ok=True)
    out = os.path.join(build, "libocomath_host.so")
    subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off", "-I",
                    os.path.join(root, "ocotillo_b200", "csrc"), "-o", out, os.path.join(root, "tests", "ocomath_host.cpp")],
                   check=True, capture_output=True)
    h = ctypes.CDLL(out)
    P = ctypes.POINTER(ctypes.c_double)
    h.exp_fast_and_dd.argtypes = [P, P, ctypes.c_int64, P, ctypes.POINTER(ctypes.c_int32), P]
    return h


def test_exp_fast_phase_equals_full_exp_where_it_succeeds(exp_host):
    """The plain kernels take the branch-free fast phase when it reports success and the full
    correctly rounded exp otherwise: wherever it succeeds it must give the same bits.  Inputs
    are double-double arguments (xl below half an ulp of xh) over the whole finite range and
    near the ends, where the fast phase must decline rather than differ."""
    import ctypes
    rng = np.random.default_rng(11)
    n = 400000
    xh = np.concatenate([rng.uniform(-745.2, 709.8, n // 2), rng.uniform(-50.0, 50.0, n // 4),
                         rng.uniform(-746.0, -700.0, n // 8), rng.uniform(700.0, 710.0, n // 8)])
    xl = xh * rng.uniform(-1.0, 1.0, xh.size) * 2.0 ** -54
    xl[::7] = 0.0
    fast, dd = np.empty_like(xh), np.empty_like(xh)
    ok = np.empty(xh.size, dtype=np.int32)
    P = ctypes.POINTER(ctypes.c_double)
    exp_host.exp_fast_and_dd(xh.ctypes.data_as(P), xl.ctypes.data_as(P), xh.size, fast.ctypes.data_as(P),
                             ok.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), dd.ctypes.data_as(P))
    good = ok.astype(bool)
    inner = np.abs(xh) <= 700.0  # the fast phase declines only toward underflow and overflow
    assert good[inner].mean() > 0.999, good[inner].mean()
    assert np.array_equal(fast[good].view(np.uint64), dd[good].view(np.uint64)), np.count_nonzero(
        fast[good].view(np.uint64) != dd[good].view(np.uint64))
