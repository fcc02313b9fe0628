"""Runs of the reference's own step loop stored in tests/golden/ref_run_*.npz
(tests/golden/make_golden.py): the oracle reproduces them bit for bit (its
RK45 controller calls libm's pow, as the reference's host build does), and the
sm_100a kernels reproduce them bit for bit through the C ABI -- every ray's
final state and every pixel of the image, RK4 and RK45 alike."""

import json

import numpy as np
import pytest

import pyoracle
from conftest import GOLDEN
from grt import abi, torus
from helpers import max_rel, run_gpu

CASES = ["c1_rk4", "c2_rk45", "c2_rk45_chunked"]


def load_case(name):
    g = np.load(GOLDEN / f"ref_run_{name}.npz")
    p = abi.Params()
    for k, v in json.loads(str(g["params"])).items():
        setattr(p, k, v)
    w = json.loads(str(g["workload"]))
    grid = torus.benchmark_torus(*w["grid"], spin=w["spin"])
    init = abi.PhotonArrays.from_dict({f: g[f"init/{f}"] for f in abi.PHOTON_FIELDS})
    final = abi.PhotonArrays.from_dict({f: g[f"final/{f}"] for f in abi.PHOTON_FIELDS})
    prod = {k.split("/", 1)[1]: g[k] for k in g.files if k.startswith("products/")}
    return p, grid, init, final, prod, w


@pytest.mark.parametrize("name", CASES)
def test_oracle_reproduces_reference_runs_bitwise(oracle, name):
    p, grid, init, final, prod, w = load_case(name)
    # the oracle's own pixel-grid initialisation equals the reference-side one
    mine = oracle.init_image_photons(p, w["pixels"], w["pixels"])
    d = pyoracle.compare_photons(mine, init)
    assert all(v == 0 for v in d.values()), d
    ph = init.copy()
    oracle.run(p, grid, ph)
    d = pyoracle.compare_photons(ph, final)
    assert all(v == 0 for v in d.values()), d
    got = oracle.image_products(p, ph)
    for f, v in prod.items():
        assert np.array_equal(getattr(got, f), v), f


@pytest.mark.parametrize("name", CASES)
def test_oracle_restated_pow_reproduces_reference_runs(oracle, name):
    """The kernels' restatement of glibc's pow, compiled for the host, gives
    the reference's runs too (the same trajectories as std::pow)."""
    p, grid, init, final, prod, w = load_case(name)
    ph = init.copy()
    oracle.set_pow_mode("restated")
    try:
        oracle.run(p, grid, ph)
    finally:
        oracle.set_pow_mode("libm")
    d = pyoracle.compare_photons(ph, final)
    assert all(v == 0 for v in d.values()), d


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_kernel_reproduces_reference_runs(gpu, name):
    p, grid, init, final, prod, w = load_case(name)
    got, gprod, _ = run_gpu(gpu, p, grid, nx=w["pixels"], ny=w["pixels"])
    # every field of every ray, bit for bit (ids, phases and flags included)
    d = pyoracle.compare_photons(got, final)
    assert all(v == 0 for v in d.values()), d
    for f in abi.PHOTON_FIELDS:
        assert np.array_equal(getattr(got, f), getattr(final, f)), f
    # per pixel: a pixel that collects several arrivals sums them in the
    # device's atomic order, so equality is to round-off, not bitwise
    assert int(gprod.arrived_count[0]) == int(prod["arrived_count"][0])
    for f in ("image_I", "image_Q", "image_U", "image_V"):
        assert max_rel(getattr(gprod, f), prod[f]) <= 1e-12, f
    assert max_rel(gprod.spectrum_I, prod["spectrum_I"]) <= 1e-12
