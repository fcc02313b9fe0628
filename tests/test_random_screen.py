"""The reference's random-screen image initialisation
(src/radiative_transfer/initialize_photons.hpp:82-170): n rays placed
uniformly on the camera plane, (u, v) = (drand(-W/2, W/2), drand(-H/2, H/2))
from a pool seeded 12345 + rank.  The product draws (u, v) from Philox keyed
by (12345 + rank, photon id) -- reproducible whatever the scheduling -- and
the oracle uses the same streams, so the two agree bit for bit (GPU test in
test_gpu_random_screen.py).  The reference's own initialiser, run here
through the shim's random pool, must agree with them in distribution: the
screen positions and the image made from them."""

import numpy as np
import pytest

from grt import config, torus, workloads
from helpers import mini

scipy_stats = pytest.importorskip("scipy.stats")


def _toml(p, w, tmp_path):
    torus.write_numpy_dir(w.torus(), tmp_path / "np")
    return config.write_toml(p, tmp_path / "c.toml", tmp_path / "np", tmp_path / "out")


def test_screen_positions_match_reference_in_distribution(oracle, reference, tmp_path):
    w = mini(workloads.C2, 16, (32, 16, 16))
    p = w.params()
    n = 20_000
    mine = oracle.init_image_photons_random(p, n, id_offset=7)
    ref = reference.init_image_photons_random(_toml(p, w, tmp_path), n, id_offset=7)
    assert np.array_equal(mine.id, ref.id)
    for a, half in ((mine.theta_disp, p.camera_width / 2), (mine.phi_disp, p.camera_height / 2)):
        assert (a >= -half).all() and (a < half).all()
        assert scipy_stats.kstest(a, scipy_stats.uniform(-half, 2 * half).cdf).pvalue > 0.01
    for f in ("theta_disp", "phi_disp"):
        assert scipy_stats.ks_2samp(getattr(mine, f), getattr(ref, f)).pvalue > 0.01, f
    # the fields that do not depend on the draw are the reference's
    for f in ("x0", "dlambda", "I", "frequency", "emission_frame_energy", "phase", "terminate"):
        assert np.array_equal(getattr(mine, f), getattr(ref, f)), f
    # the draws are independent of each other and of the photon index
    assert abs(np.corrcoef(mine.theta_disp, mine.phi_disp)[0, 1]) < 0.05
    assert abs(np.corrcoef(mine.theta_disp, np.arange(n))[0, 1]) < 0.05


def test_random_screen_image_matches_reference_in_distribution(oracle, reference, tmp_path):
    w = mini(workloads.C2, 16, (32, 16, 16))
    p = w.params()
    n = 6000
    toml = _toml(p, w, tmp_path)
    mine = oracle.init_image_photons_random(p, n)
    oracle.run(p, w.torus(), mine)
    ref = reference.init_image_photons_random(toml, n)
    reference.run(toml, ref, p)
    a_mine, a_ref = mine.phase == 3, ref.phase == 3
    # arrived fractions agree within binomial noise
    f1, f2 = a_mine.mean(), a_ref.mean()
    sigma = np.sqrt(f1 * (1 - f1) / n + f2 * (1 - f2) / n)
    assert abs(f1 - f2) <= 4 * sigma + 1e-12, (f1, f2)
    # arrival positions and intensities agree in distribution
    for f in ("theta_disp", "phi_disp", "I"):
        assert scipy_stats.ks_2samp(getattr(mine, f)[a_mine], getattr(ref, f)[a_ref]).pvalue > 0.01, f
