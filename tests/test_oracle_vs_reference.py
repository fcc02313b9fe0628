"""The oracle against the reference's own code (compiled from the reference
tree against oracle/shim): with the controller's pow taken from libm, exactly
like the reference's host build, every field of every ray is bit-identical,
and so it is with the kernels' restatement of glibc's pow in its place."""

import numpy as np
import pytest

import pyoracle
from grt import config, workloads
from helpers import mini

CASES = [mini(workloads.C1, 12, (24, 16, 16)), mini(workloads.C2, 16, (32, 16, 16)),
         mini(workloads.C2, 12, (24, 12, 12), integrator=0, initial_step=0.002, max_steps=1200)]


def _run_both(reference, oracle, w, tmp_path):
    p = w.params()
    grid = w.torus()
    from grt import torus
    torus.write_numpy_dir(grid, tmp_path / "np")
    toml = config.write_toml(p, tmp_path / "c.toml", tmp_path / "np", tmp_path / "out")
    ref_ph = reference.init_image_photons(toml, w.pixels, w.pixels)
    ora_ph = oracle.init_image_photons(p, w.pixels, w.pixels)
    init_diff = pyoracle.compare_photons(ref_ph, ora_ph)
    assert all(v == 0 for v in init_diff.values()), init_diff
    ref_prod, ref_stats = reference.run(toml, ref_ph, p)
    return p, grid, ora_ph, ref_ph, ref_prod, ref_stats


@pytest.mark.parametrize("w", CASES, ids=["c1_rk4", "c2_rk45", "rk4_24px"])
def test_oracle_libm_bit_identical_to_reference(reference, oracle, w, tmp_path):
    p, grid, ora_ph, ref_ph, ref_prod, ref_stats = _run_both(reference, oracle, w, tmp_path)
    st = oracle.run(p, grid, ora_ph)
    d = pyoracle.compare_photons(ref_ph, ora_ph)
    assert all(v == 0 for v in d.values()), d
    prod = oracle.image_products(p, ora_ph)
    for f in ("image_I", "image_Q", "image_U", "image_V", "spectrum_I", "spectrum_frequency_hz", "arrived_count"):
        assert np.array_equal(getattr(prod, f), getattr(ref_prod, f)), f
    # the shim counts the functor's stepping invocations
    assert st["accepted_steps"] == ref_stats["stepped"]


def test_oracle_restated_pow_bit_identical_to_reference(reference, oracle, tmp_path):
    w = CASES[1]
    p, grid, ora_ph, ref_ph, ref_prod, _ = _run_both(reference, oracle, w, tmp_path)
    oracle.set_pow_mode("restated")
    try:
        oracle.run(p, grid, ora_ph)
    finally:
        oracle.set_pow_mode("libm")
    d = pyoracle.compare_photons(ref_ph, ora_ph)
    assert all(v == 0 for v in d.values()), d
