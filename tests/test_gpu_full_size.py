"""Parity at the full sizes of the benchmark configurations, where rare
events -- a ray that grazes a cell's acceptance boundary, a controller input
near a rounding tie, a long path -- have room to happen:

* C1: 64x64 rays, RK4, 64x32x32 torus, a = 0.9, 60 deg;
* C2: 256x256 rays, RK45 rtol = atol = 1e-8, 128x64x64 torus, a = 0.94,
  17 deg, FP64 form;
* one 512x512 image of the C3 batch (128x64x64 torus, a = 0.9, RK45) at its
  inclination and frequency channel.

Each is compared ray by ray, every field bit for bit, with the oracle (whose
controller calls glibc's pow, as the reference's host build does), and C1 and
C2 also with the reference's own step loop (oracle/_ref) and its image
products per pixel.  Pixels that collect several arrivals are summed in the
device's atomic order, so images agree to round-off rather than bitwise."""

import math

import numpy as np
import pytest

import pyoracle
from grt import config, torus, workloads
from helpers import FP64_RTOL, max_rel, run_gpu

pytestmark = pytest.mark.gpu

PRODUCT_FIELDS = ("image_I", "image_Q", "image_U", "image_V", "spectrum_I")


def assert_bitwise(got, want):
    d = pyoracle.compare_photons(got, want)
    assert all(v == 0 for v in d.values()), d


def assert_products(got, want):
    assert int(got.arrived_count[0]) == int(want.arrived_count[0])
    # image pixels collect a few arrivals each; a spectrum bin collects
    # thousands, summed by device atomics in another order than the
    # reference's serial loop, so it is held to the 1e-9 parity bar
    for f in PRODUCT_FIELDS:
        tol = FP64_RTOL if f == "spectrum_I" else 1e-12
        assert max_rel(getattr(got, f), getattr(want, f)) <= tol, f


@pytest.mark.parametrize("w", [workloads.C1, workloads.C2], ids=["c1_rk4_64px", "c2_rk45_256px"])
def test_full_size_image_matches_oracle_and_reference(gpu, oracle, reference, w, tmp_path):
    p = w.params()
    grid = w.torus()
    got, gprod, st = run_gpu(gpu, p, grid, nx=w.pixels, ny=w.pixels)
    assert st["timed_out"] == 0
    ph = oracle.init_image_photons(p, w.pixels, w.pixels)
    oracle.run(p, grid, ph)
    assert_bitwise(got, ph)
    assert_products(gprod, oracle.image_products(p, ph))
    # the reference's own step loop and products on the same config
    torus.write_numpy_dir(grid, tmp_path / "np")
    toml = config.write_toml(p, tmp_path / "c.toml", tmp_path / "np", tmp_path / "out")
    ref_ph = reference.init_image_photons(toml, w.pixels, w.pixels)
    ref_prod, _ = reference.run(toml, ref_ph, p)
    assert_bitwise(got, ref_ph)
    assert_products(gprod, ref_prod)


def test_c3_512px_image_matches_oracle(gpu, oracle):
    incl, px, f_ghz = next(im for im in workloads.C3.images if im[1] == 512)
    base = workloads.C3.base
    w = workloads.ImageWorkload("c3_512px", base.grid, base.spin, incl, px, base.integrator, base.initial_step,
                                base.max_steps,
                                extra=dict(custom_frequency_hz=f_ghz * 1e9, emission_coefficient=f_ghz / 230.0))
    p = w.params()
    assert math.isclose(p.camera_theta, math.radians(incl))
    grid = w.torus()
    got, gprod, st = run_gpu(gpu, p, grid, nx=px, ny=px)
    assert st["timed_out"] == 0
    ph = oracle.init_image_photons(p, px, px)
    oracle.run(p, grid, ph)
    assert_bitwise(got, ph)
    assert_products(gprod, oracle.image_products(p, ph))
    assert np.count_nonzero(gprod.image_I) > 1000
