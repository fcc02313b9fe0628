"""The oracle against the known answers of the reference's own unit tests
(src/tests/*.cpp) and against values of reference functions stored in
tests/golden/ref_known_answers.npz (tests/golden/make_golden.py)."""

import ctypes as C
import math

import numpy as np
import pytest

from conftest import GOLDEN
from grt import abi, workloads
from grt.config import reference_defaults

_DP = C.POINTER(C.c_double)


def dp(a):
    return a.ctypes.data_as(_DP)


@pytest.fixture(scope="module")
def ka():
    return np.load(GOLDEN / "ref_known_answers.npz")


@pytest.mark.parametrize("a", [1.0, 0.9, 0.94])
def test_rhs_and_null_momentum_match_reference_functions(oracle, ka, a):
    X, K = ka["X"], ka["K"]
    ok, P = oracle.null_momentum(X, K, a, 1.0)
    assert ok
    assert np.array_equal(P, ka[f"a{a}/null_p"])
    assert np.array_equal(oracle.rhs(X, P, a, 1.0), ka[f"a{a}/rhs"])
    # null norm below 1e-10 (src/tests/test_geodesic_observables.cpp:37-45)
    assert abs(oracle.lib.oracle_norm(dp(X), dp(P), a, 1.0)) < 1e-10
    assert abs(ka[f"a{a}/observables"][0]) < 1e-10


@pytest.mark.parametrize("a", [1.0, 0.9])
def test_rhs_equals_explicit_metric_derivative_contraction(oracle, a):
    # test_geodesic_observables.cpp:47-66: dx^mu = g^{mu nu} p_nu and
    # dp_mu = -1/2 d_mu g^{ab} p_a p_b, to 1e-12.
    X = np.array([0.0, 5.0, -7.0, 2.0])
    ok, P = oracle.null_momentum(X, [0.4, -0.5, 0.768], a, 1.0)
    rhs = oracle.rhs(X, P, a, 1.0)
    g = np.zeros(16); d = np.zeros(64)
    oracle.lib.oracle_inverse_metric(dp(X), a, 1.0, dp(g))
    oracle.lib.oracle_inverse_metric_deriv(dp(X), a, 1.0, dp(d))
    g = g.reshape(4, 4); d = d.reshape(4, 4, 4)
    for mu in range(4):
        assert abs(rhs[mu] - g[mu] @ P) < 1e-12
        assert abs(rhs[4 + mu] + 0.5 * P @ d[mu] @ P) < 1e-12


def _params(**kw):
    p = reference_defaults()
    p.update(**kw)
    return p


def test_rk_steps_exact_on_straight_lines(oracle):
    # test_rk_integrators.cpp: RK4/RK45 are exact for linear motion; with
    # M = 0 the photon ODE is x' = p, p' = 0.
    p = _params(mass=1e-300, spin=0.0)
    s = np.array([0.0, 10.0, -3.0, 2.0, -1.0, 0.6, 0.0, -0.8])
    s4 = s.copy()
    oracle.lib.oracle_rk4_step(C.byref(p), dp(s4), 0.5)
    assert np.allclose(s4[1:4], s[1:4] + 0.5 * s[5:8], rtol=0, atol=1e-14)
    s45 = s.copy()
    dl = np.array([0.5])
    assert oracle.lib.oracle_rk45_step(C.byref(p), dp(s45), dp(dl)) == 1
    assert np.allclose(s45[1:4], s[1:4] + 0.5 * s[5:8], rtol=0, atol=1e-14)


def test_rk4_converges_at_fourth_order(oracle):
    # test_convergence.cpp:62-83: Kerr geodesic from X = (0, 6, 2, 1), direction
    # (-0.4, 0.8, 0.2), interval 4; error ratio > 10 on halving the step.
    p = _params(spin=1.0, mass=1.0)
    ok, P = oracle.null_momentum([0.0, 6.0, 2.0, 1.0], [-0.4, 0.8, 0.2], 1.0, 1.0)
    s0 = np.array([0.0, 6.0, 2.0, 1.0, *P])

    def integrate(n):
        s = s0.copy()
        for _ in range(n):
            oracle.lib.oracle_rk4_step(C.byref(p), dp(s), 4.0 / n)
        return s
    ref = integrate(8192)
    e8, e16, e32 = (np.max(np.abs(integrate(n) - ref)) for n in (8, 16, 32))
    assert e8 / e16 > 10.0 and e16 / e32 > 10.0


@pytest.mark.parametrize("case", ["absorb", "emit", "off", "negative_path", "vacuum"])
def test_radiative_transfer_cases(oracle, case):
    # test_radiative_transfer.cpp:14-79
    st = np.array([4.0, 2.0, 1.0, 0.5])
    e = math.exp(-1.0)
    if case == "absorb":
        oracle.lib.oracle_apply_rt(dp(st), 1.0, 2.0, 1e14, 1.0, 1, 0, 1.0, 0.0)
        assert np.allclose(st, [4 * e, 2 * e, e, 0.5 * e], rtol=0, atol=1e-12)
    elif case == "emit":
        oracle.lib.oracle_apply_rt(dp(st), 1.0, 2.0, 1e14, 1.0, 0, 1, 0.0, 1.0)
        assert abs(st[0] - 6.0) < 1e-12 and list(st[1:]) == [2.0, 1.0, 0.5]
    elif case == "off":
        oracle.lib.oracle_apply_rt(dp(st), 1.0, 2.0, 1e14, 1.0, 0, 0, 0.0, 0.0)
        assert list(st) == [4.0, 2.0, 1.0, 0.5]
    elif case == "negative_path":
        st = np.array([4.0, 0.0, 0.0, 0.0])
        oracle.lib.oracle_apply_rt(dp(st), 1.0, 2.0, 1e14, -1.0, 1, 0, 1.0, 0.0)
        assert abs(st[0] - 4 * e) < 1e-12
    else:
        oracle.lib.oracle_apply_rt(dp(st), 0.0, 5.0, 1e14, 1.0, 1, 1, 10.0, 10.0)
        assert abs(st[0] - 4.0) < 1e-12 and list(st[1:]) == [2.0, 1.0, 0.5]


def test_nonuniform_lookup_known_cell_and_random_queries(oracle, ka):
    # test_npy_loader.cpp:74-97: the centre of cell (2, 1, 3) of a fully 3-D
    # nonuniform grid is located at (2, 1, 3); plus 200 random queries
    # answered by the reference's own locate_structured_grid_cell.
    from make_golden import npy_loader_grid
    r, th, ph = npy_loader_grid()
    ok, ijk = oracle.locate_cell(r, th, ph, r[2, 1, 3], th[2, 1, 3], ph[2, 1, 3])
    assert ok and ijk == (2, 1, 3)
    assert list(ka["npy_loader/located"]) == [1, 2, 1, 3]
    for row in ka["npy_loader/random_queries"]:
        ok, ijk = oracle.locate_cell(r, th, ph, *row[:3])
        assert int(ok) == int(row[3])
        if ok:
            assert ijk == tuple(int(v) for v in row[4:])


def test_observation_products_known_answer(oracle):
    # test_output_stride.cpp:19-45: one ImageArrived photon with I = 2 and one
    # Rejected photon with I = 100 give arrived_count 1 and an image sum of 2.
    p = _params(image_nx=4, image_ny=4, spectrum_bins=8, spectrum_min_hz=1e9, spectrum_max_hz=1e15,
                camera_width=20.0, camera_height=20.0)
    ph = abi.PhotonArrays(2)
    ph.frequency[:] = 1e12
    ph.I[:] = [2.0, 100.0]
    ph.phase[:] = [abi.PHASE_ARRIVED, abi.PHASE_REJECTED]
    prod = oracle.image_products(p, ph)
    assert int(prod.arrived_count[0]) == 1 and prod.image_I.sum() == 2.0


def test_observation_bin_edges(oracle):
    # observation.hpp:22-29 bins with floor(clamp(frac) * (bins - 1)): the top
    # edge falls into the last bin and out-of-range values are clamped.
    b = oracle.lib.oracle_observation_bin
    assert b(-10.0, -1.0, 1.0, 4) == 0 and b(1.0, -1.0, 1.0, 4) == 3 and b(5.0, -1.0, 1.0, 4) == 3
    assert b(0.999, -1.0, 1.0, 4) == 2 and b(0.3, 1.0, 1.0, 4) == 0 and b(0.3, -1.0, 1.0, 1) == 0


def test_philox_known_answers(oracle):
    # Philox4x32-10 test vectors published with the Random123 library.
    def block(ctr, key):
        c = (C.c_uint32 * 4)(*ctr)
        k = (C.c_uint32 * 2)(*key)
        o = (C.c_uint32 * 4)()
        oracle.lib.oracle_philox_block(c, k, o)
        return list(o)
    assert block([0, 0, 0, 0], [0, 0]) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert block([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    assert block([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0]) == \
        [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]
    d = [oracle.lib.oracle_philox_drand(12345, 7, 3, i) for i in range(6)]
    assert all(0.0 <= x < 1.0 for x in d) and len(set(d)) == 6
