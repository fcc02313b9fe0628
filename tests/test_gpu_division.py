"""The FP64 right-hand side forms its 21 quotients from six correctly rounded
reciprocals and Markstein's residual corrections (grt_div.cuh, ks_rhs_rcp)
whenever the state lies in a box where no value under- or overflows, and
uses IEEE divisions outside it.  The parity form is bit-exact only if every
such quotient equals the IEEE quotient, so this checks, on the GPU, through
lib/libgrt_selftest.so (built from the same headers with the same flags as
the trace kernels):

* div_by against CUDA's IEEE a / b, bit for bit, on random operands over a
  wide exponent span, on quotients within half an ulp of a rounding
  midpoint, and on signed zeros;
* ks_rhs_rcp against ks_rhs (IEEE divisions), all seven components bit for
  bit, on random photon states from the horizon to 2000 M, with exactly zero
  coordinates, for several spins; states outside the box (coordinates of
  magnitude below 2^-20 or above 2^20) must be reported outside;
* the RK45 controller's pow_quarter on the device against this host's glibc
  pow(x, 0.25), bit for bit, on tie-near inputs (tests/golden/pow_quarter_hard.npz)
  and on random inputs over the controller's range and over all doubles;
* the branch-free reciprocal and square root of the image-mode kernels
  (grt_rn.cuh) against CUDA's __drcp_rn and sqrt, bit for bit, on random
  arguments over their exact ranges ([2^-1000, 2^1000] for the reciprocal,
  [2^-900, 2^1000] for the square root), significands near all ones and near one,
  and arguments next to squares of rounding midpoints; and ks_rhs_rcp with
  them against ks_rhs_rcp with CUDA's, components and box flag."""

import ctypes as C
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LIB = Path(__file__).resolve().parent.parent / "gr-ray-tracer_b200" / "lib" / "libgrt_selftest.so"
_DP = C.POINTER(C.c_double)
_UP = C.POINTER(C.c_uint32)


@pytest.fixture(scope="module")
def selftest(gpu):
    if not LIB.exists():
        pytest.fail(f"{LIB} is missing (make -C gr-ray-tracer_b200)")
    L = C.CDLL(str(LIB))
    L.grt_selftest_division.argtypes = [_DP, _DP, C.c_size_t, _DP, _DP]
    L.grt_selftest_rhs.argtypes = [_DP, C.c_size_t, C.c_double, C.c_double, _DP, _DP, _UP]
    L.grt_selftest_pow_quarter.argtypes = [_DP, C.c_size_t, _DP]
    L.grt_selftest_rn_box.argtypes = [_DP, C.c_size_t, _DP, _DP, _DP, _DP]
    L.grt_selftest_rhs_bf.argtypes = [_DP, C.c_size_t, C.c_double, C.c_double, _DP, _DP, _UP]
    return L


def dp(a):
    return a.ctypes.data_as(_DP)


def divide(L, a, b):
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    q, w = np.empty(a.size), np.empty(a.size)
    assert L.grt_selftest_division(dp(a), dp(b), a.size, dp(q), dp(w)) == 0
    return q, w


def random_doubles(rng, n, emin, emax):
    mant = rng.random(n) + 1.0
    e = rng.integers(emin, emax, n)
    sign = np.where(rng.random(n) < 0.5, -1.0, 1.0)
    return sign * np.ldexp(mant, e)


def assert_bitwise(q, w, mask=None):
    qi, wi = q.view(np.int64), w.view(np.int64)
    if mask is not None:
        qi, wi, q, w = qi[mask], wi[mask], q[mask], w[mask]
    bad = np.flatnonzero(qi != wi)
    assert bad.size == 0, (bad.size, q[bad[:5]], w[bad[:5]])


def test_random_quotients_are_ieee(selftest):
    rng = np.random.default_rng(11)
    n = 1 << 22
    a = random_doubles(rng, n, -450, 450)
    b = random_doubles(rng, n, -450, 450)
    assert_bitwise(*divide(selftest, a, b))
    # denominators with mantissas near 1 and near 2
    b2 = np.ldexp(1.0 + rng.random(n) * 2.0 ** -20, rng.integers(-40, 40, n))
    b3 = np.ldexp(2.0 - rng.random(n) * 2.0 ** -20, rng.integers(-40, 40, n))
    for bb in (b2, b3):
        assert_bitwise(*divide(selftest, a * 2.0 ** -400, bb))


def test_near_midpoint_quotients_are_ieee(selftest):
    # a = RN(b * m), m the midpoint between q and its successor: a / b lies
    # within about half an ulp of a rounding boundary; a's neighbours move
    # it across
    rng = np.random.default_rng(12)
    n = 1 << 21
    q0 = np.abs(random_doubles(rng, n, -200, 200))
    b = random_doubles(rng, n, -200, 200)
    m = q0.astype(np.longdouble) + (np.nextafter(q0, np.inf) - q0).astype(np.longdouble) / 2
    a = (np.asarray(b, dtype=np.longdouble) * m).astype(np.float64)
    for aa in (a, np.nextafter(a, np.inf), np.nextafter(a, -np.inf)):
        assert_bitwise(*divide(selftest, aa, b))


def test_zero_numerators_keep_their_sign(selftest):
    assert_bitwise(*divide(selftest, np.array([0.0, -0.0, 0.0, -0.0]), np.array([3.0, 3.0, -3.0, -3.0])))


def random_states(rng, n, spin):
    """Photon states (x, y, z, p_t, p_x, p_y, p_z) with Kerr-Schild radius
    from just outside the horizon to 2000 M."""
    r_h = 1.0 + np.sqrt(max(0.0, 1.0 - spin * spin))
    r = np.exp(rng.uniform(np.log(1.02 * r_h), np.log(2000.0), n))
    ct = rng.uniform(-1.0, 1.0, n)
    ph = rng.uniform(0.0, 2 * np.pi, n)
    st = np.sqrt(1.0 - ct * ct)
    x = (r * np.cos(ph) - spin * np.sin(ph)) * st
    y = (r * np.sin(ph) + spin * np.cos(ph)) * st
    z = r * ct
    k = rng.normal(size=(n, 3))
    k /= np.linalg.norm(k, axis=1)[:, None]
    s = np.column_stack([x, y, z, -np.ones(n), k * rng.uniform(0.5, 2.0, (n, 1))])
    q = n // 8
    s[:q, 2] = 0.0            # equatorial plane
    s[q:2 * q, 0] = 0.0       # x = 0 plane
    s[2 * q:3 * q, 1] = 0.0   # y = 0 plane
    s[3 * q:4 * q, 5] = 0.0   # a zero momentum component
    s[4 * q:4 * q + 64, 0] = -0.0
    return np.ascontiguousarray(s)


def rhs(L, s, spin, M=1.0):
    n = s.shape[0]
    fast, ieee = np.empty((n, 7)), np.empty((n, 7))
    inside = np.empty(n, dtype=np.uint32)
    assert L.grt_selftest_rhs(dp(s), n, spin, M, dp(fast), dp(ieee), inside.ctypes.data_as(_UP)) == 0
    return fast, ieee, inside.astype(bool)


@pytest.mark.parametrize("spin", [0.0, 0.5, 0.9, 0.94, 0.999, 1.0, -0.7])
def test_rhs_with_reciprocals_is_ieee_rhs(selftest, spin):
    rng = np.random.default_rng(int(abs(spin) * 1000) + 13)
    s = random_states(rng, 1 << 19, spin)
    fast, ieee, inside = rhs(selftest, s, spin)
    assert inside.mean() > 0.99, inside.mean()
    assert_bitwise(fast.ravel(), ieee.ravel(), np.repeat(inside, 7))


def test_states_outside_the_box_are_reported(selftest):
    s = np.tile(np.array([[10.0, -20.0, 5.0, -1.0, 0.3, -0.5, 0.8]]), (6, 1))
    s[0, 0] = 2.0 ** -21       # below 2^-20
    s[1, 1] = -(2.0 ** 21)     # above 2^20
    s[2, 2] = np.nan
    s[3, 0] = 5e-324           # subnormal
    # inside: exact zeros and the box's edges
    s[4, 0] = 0.0
    s[5, 0] = 2.0 ** -20
    _, _, inside = rhs(selftest, s, 0.9)
    assert inside.tolist() == [False, False, False, False, True, True]


def test_device_pow_quarter_is_glibc_pow(selftest, oracle):
    from conftest import GOLDEN
    g = np.load(GOLDEN / "pow_quarter_hard.npz")
    rng = np.random.default_rng(17)
    xs = [g["x_controller"], g["x_wide"], np.exp(rng.uniform(np.log(1.5e-8), np.log(2e4), 4_000_000)),
          rng.integers(0, 0x7FF0000000000000, 1_000_000, dtype=np.uint64).view(np.float64),
          np.array([0.0, -0.0, np.inf, -np.inf, 5e-324, 2.0 ** -1022, 1.0, 1.0 + 2.0 ** -52, 1.0 - 2.0 ** -53])]
    x = np.ascontiguousarray(np.concatenate(xs))
    y = np.empty_like(x)
    assert selftest.grt_selftest_pow_quarter(dp(x), x.size, dp(y)) == 0
    want, host = np.empty_like(x), np.empty_like(x)  # std::pow (glibc) and the host build
    oracle.lib.oracle_pow_quarter_pair(x.ctypes.data, C.c_uint64(x.size), want.ctypes.data, host.ctypes.data)
    assert_bitwise(y, want)
    assert_bitwise(host, want)
    assert np.array_equal(y[: g["x_controller"].size], g["pow_controller"])


def rn_box(L, x):
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = [np.empty(x.size) for _ in range(4)]
    assert L.grt_selftest_rn_box(dp(x), x.size, *(dp(o) for o in out)) == 0
    return out


def test_branch_free_reciprocal_and_sqrt_are_cudas(selftest):
    rng = np.random.default_rng(19)
    n = 1 << 22
    e = rng.integers(-1000, 1000, n)
    sign = np.where(rng.random(n) < 0.5, -1.0, 1.0)
    random = sign * np.ldexp(1.0 + rng.integers(0, 1 << 52, n, dtype=np.int64) * 2.0 ** -52, e)
    k = rng.integers(0, 1 << 16, n)
    near_two = sign * np.ldexp(2.0 - k * 2.0 ** -52, e)     # all ones at k = 1
    near_one = sign * np.ldexp(1.0 + k * 2.0 ** -52, e)
    ones = np.ldexp(2.0 - 2.0 ** -52, np.arange(-999, 1000))  # every all-ones significand's exponent
    edges = np.array([2.0 ** -1000, 2.0 ** -900, 2.0 ** 1000, 1.0, 2.0, 3.0, 0.5, 1.0 + 2.0 ** -52,
                      2.0 - 2.0 ** -51])
    for x in (random, near_two, near_one, np.concatenate([ones, -ones, edges, -edges])):
        rb, rc, sb, sc = rn_box(selftest, x)
        assert_bitwise(rb, rc)
        assert_bitwise(sb, sc, np.abs(x) >= 2.0 ** -900)
    # next to squares of midpoints: sqrt lies within a tiny fraction of an
    # ulp of a rounding boundary
    m = np.ldexp(1.0 + rng.integers(0, 1 << 52, n // 8, dtype=np.int64) * 2.0 ** -52, rng.integers(-449, 490, n // 8))
    ulp = np.nextafter(m, np.inf) - m
    v = m * m + m * ulp
    for d in range(-3, 4):
        w = v.view(np.int64) + d
        _, _, sb, sc = rn_box(selftest, w.view(np.float64))
        assert_bitwise(sb, sc)


def test_branch_free_outside_arguments_fail_the_box(selftest):
    # zero, subnormal, infinity and NaN give NaN from the square root, which
    # fails ks_rhs_rcp's box check as CUDA's out-of-box results do; below
    # 2^-900 the result stays below 2^-450, far outside the box
    x = np.array([0.0, 5e-324, 2.0 ** -1060, np.inf, np.nan])
    _, _, sb, _ = rn_box(selftest, x)
    assert np.isnan(sb).all(), sb
    rng = np.random.default_rng(29)
    low = np.ldexp(1.0 + rng.random(1 << 16), rng.integers(-1022, -900, 1 << 16))
    _, _, sb, sc = rn_box(selftest, low)
    assert (sb < 2.0 ** -449).all() and (np.abs(sb - sc) <= np.spacing(sc)).all()


def rhs_bf(L, s, spin, M=1.0):
    n = s.shape[0]
    bf, ref = np.empty((n, 7)), np.empty((n, 7))
    inside = np.empty(n, dtype=np.uint32)
    assert L.grt_selftest_rhs_bf(dp(s), n, spin, M, dp(bf), dp(ref), inside.ctypes.data_as(_UP)) == 0
    return bf, ref, inside


@pytest.mark.parametrize("spin", [0.0, 0.94, 1.0, -0.7])
def test_branch_free_rhs_is_the_rhs(selftest, spin):
    rng = np.random.default_rng(int(abs(spin) * 1000) + 23)
    s = random_states(rng, 1 << 19, spin)
    out = np.tile(np.array([[10.0, -20.0, 5.0, -1.0, 0.3, -0.5, 0.8]]), (5, 1))
    out[0, 0] = 2.0 ** -21
    out[1, 1] = -(2.0 ** 21)
    out[2, 2] = np.nan
    out[3, 0] = 5e-324
    out[4, :3] = [spin, 0.0, 0.0]   # on the ring: S = 0
    s = np.ascontiguousarray(np.vstack([s, out]))
    bf, ref, inside = rhs_bf(selftest, s, spin)
    ok_bf, ok_ref = (inside & 1).astype(bool), (inside & 2).astype(bool)
    assert np.array_equal(ok_bf, ok_ref)
    assert ok_bf.mean() > 0.99
    assert not ok_bf[-5:].any()
    assert_bitwise(bf.ravel(), ref.ravel(), np.repeat(ok_ref, 7))
