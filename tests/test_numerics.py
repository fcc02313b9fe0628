"""Pinned numerics of the oracle: the algorithmic op counts the roofline uses
and the correctly rounded fourth root of the RK45 controller."""

import ctypes as C
import math
import random

import numpy as np
import pytest

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


def test_fourth_root_correctly_rounded(oracle):
    mpmath = pytest.importorskip("mpmath")
    mpmath.mp.prec = 300
    random.seed(11)
    xs = [10 ** random.uniform(-300, 300) for _ in range(4000)]
    xs += [10 ** random.uniform(-12, 8) for _ in range(4000)]
    xs += [5e-324, 1e-310, 2.0 ** -1022, 1.0, 16.0, 0.5, 2.0, 1.7976931348623157e308]
    for x in xs:
        want = float(mpmath.mpf(x) ** mpmath.mpf(0.25))
        assert oracle.lib.oracle_fourth_root(x) == want, x
    assert oracle.lib.oracle_fourth_root(0.0) == 0.0
    assert math.isinf(oracle.lib.oracle_fourth_root(math.inf))


def test_product_fourth_root_matches_oracle(oracle):
    """The kernels' fourth_root_cr (rounding test with a 256-bit fallback),
    compiled for the host, equals the oracle's arbitrary-precision root bit for
    bit -- on random inputs over the whole range, on fourth powers of rounding
    midpoints and their neighbours (the hardest cases), and around powers of two."""
    rng = np.random.default_rng(1)
    y = 10.0 ** rng.uniform(-200, 200, 500_000)
    mids = y + np.spacing(y) / 2
    with np.errstate(over="ignore"):
        m4 = mids ** 4
        cases = [m4, np.nextafter(m4, np.inf), np.nextafter(m4, 0.0), y ** 4,
                 10.0 ** rng.uniform(-300, 300, 500_000), 10.0 ** rng.uniform(-12, 8, 500_000)]
    p2 = np.ldexp(1.0, rng.integers(-1070, 1020, 50_000))
    cases += [p2, np.nextafter(p2, 0.0), np.nextafter(p2, np.inf),
              np.array([5e-324, 1e-310, 2.0 ** -1022, 2.0 ** -900, 2.0 ** 900, 1.7976931348623157e308])]
    x = np.concatenate(cases)
    x = np.ascontiguousarray(x[np.isfinite(x) & (x > 0)])
    a = np.empty_like(x)
    b = np.empty_like(x)
    oracle.lib.oracle_fourth_root_pair(x.ctypes.data, C.c_uint64(x.size), a.ctypes.data, b.ctypes.data)
    bad = np.flatnonzero(a.view(np.uint64) != b.view(np.uint64))
    assert bad.size == 0, x[bad[:5]]


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
