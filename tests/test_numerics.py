"""Pinned numerics: the algorithmic op counts the roofline uses, the RK45
controller's pow(x, 0.25) against glibc's, and the deterministic sin/cos."""

import ctypes as C
import math
import random

import numpy as np
import pytest

from conftest import GOLDEN
from grt import workloads

_DP = C.POINTER(C.c_double)


def test_op_counts_pinned(oracle):
    # One RHS = 243 ops, one RK4 step = 1100, one RKF45 attempt (k1 given) =
    # 1691, counted over the reference's source operations (add/sub, mul, div,
    # sqrt, pow each 1) by a counting scalar type that reproduces the double
    # results exactly (checks == 0).
    import bench
    p = workloads.C2.params()
    ok, P = oracle.null_momentum([0.0, 6.0, 2.0, 1.0], [-0.4, 0.8, 0.2], p.spin, p.mass)
    X = np.array([0.0, 6.0, 2.0, 1.0])
    a = (C.c_uint64 * 5)(); b = (C.c_uint64 * 5)(); c = (C.c_uint64 * 5)(); ch = (C.c_double * 3)()
    oracle.lib.oracle_op_counts(C.byref(p), X.ctypes.data_as(_DP), P.ctypes.data_as(_DP), C.c_double(0.3),
                                a, b, c, ch)
    assert list(ch) == [0.0, 0.0, 0.0]
    assert sum(a) == bench.OPS_RHS == 243
    assert sum(b) == bench.OPS_RK4_STEP == 1100
    assert sum(c) == bench.OPS_RK45_ATTEMPT == 1691
    assert list(a) == [61, 159, 21, 2, 0]


def _pow_pair(oracle, x):
    x = np.ascontiguousarray(x, dtype=np.float64)
    libm = np.empty_like(x)
    mine = np.empty_like(x)
    oracle.lib.oracle_pow_quarter_pair(x.ctypes.data, C.c_uint64(x.size), libm.ctypes.data, mine.ctypes.data)
    return libm, mine


def _assert_bitwise(x, a, b):
    same = (a.view(np.uint64) == b.view(np.uint64)) | (np.isnan(a) & np.isnan(b))
    bad = np.flatnonzero(~same)
    assert bad.size == 0, [(float(x[i]).hex(), float(a[i]).hex(), float(b[i]).hex()) for i in bad[:5]]


def test_pow_quarter_matches_glibc_on_tie_near_inputs(oracle):
    """The kernels' controller root grt::pow_quarter (compiled for the host)
    returns glibc's pow(x, 0.25) bit for bit on inputs whose exact root lies
    within 2^-14 ulp of a rounding tie -- where a pow that is not correctly
    rounded can round either way (tests/golden/make_pow_hard.py).  The stored
    outputs are glibc's from the machine that wrote the fixture; this host's
    std::pow must give the same, or the reference itself would round
    differently here."""
    g = np.load(GOLDEN / "pow_quarter_hard.npz")
    for part in ("controller", "wide"):
        x, want = g[f"x_{part}"], g[f"pow_{part}"]
        assert x.size > 1000
        libm, mine = _pow_pair(oracle, x)
        _assert_bitwise(x, libm, want)
        _assert_bitwise(x, mine, want)


def test_pow_quarter_matches_glibc_on_random_inputs(oracle):
    """Random inputs over the controller's unclamped range, over all positive
    doubles (subnormals, powers of two and values next to 1 included), and the
    special values 0, inf, NaN and negatives."""
    rng = np.random.default_rng(7)
    ctrl = np.exp(rng.uniform(np.log(1.5e-8), np.log(2e4), 3_000_000))
    allpos = rng.integers(0, 0x7FF0000000000000, 1_000_000, dtype=np.uint64).view(np.float64)
    p2 = np.ldexp(1.0, rng.integers(-1074, 1023, 20_000))
    near1 = 1.0 + rng.integers(-2000, 2000, 20_000) * 2.0 ** -52
    special = np.array([0.0, -0.0, np.inf, -np.inf, np.nan, -1.0, 5e-324, 2.0 ** -1022, 1.7976931348623157e308])
    x = np.concatenate([ctrl, allpos, p2, np.nextafter(p2, 0.0), np.nextafter(p2, np.inf), near1, special])
    libm, mine = _pow_pair(oracle, x)
    _assert_bitwise(x, libm, mine)


def test_deterministic_sincos_accuracy(oracle):
    """grt_sincos.h (scattering and emission directions, shared by the kernels
    and the oracle): within 1.2e-16 absolute of sin/cos on [0, 2 pi], and at
    most 1 ulp where |value| > 1e-3 (mpmath at 120 bits on a sample)."""
    mpmath = pytest.importorskip("mpmath")
    mpmath.mp.prec = 120
    rng = np.random.default_rng(5)
    x = np.concatenate([rng.uniform(0.0, 2.0 * np.pi, 4000),
                        np.array([0.0, np.pi / 4, np.pi / 2, np.pi, 1.5 * np.pi, 2.0 * np.pi - 1e-12])])
    s = np.empty_like(x)
    c = np.empty_like(x)
    oracle.lib.oracle_det_sincos(x.ctypes.data, C.c_uint64(x.size), s.ctypes.data, c.ctypes.data)
    for xi, si, ci in zip(x, s, c):
        for got, want in ((si, float(mpmath.sin(xi))), (ci, float(mpmath.cos(xi)))):
            assert abs(got - want) <= 1.2e-16, (xi, got, want)
            if abs(want) > 1e-3:
                assert abs(got - want) <= np.spacing(abs(want)), (xi, got, want)
