"""The FP64 reference gradient (oracle) of a Stokes-I image loss with respect
to the per-cell absorption/emission multipliers, checked against central
finite differences of the oracle's own forward runs (CPU only).  The image is
made of line-of-sight forward rays, as in the adjoint workload."""

import numpy as np
import pytest

from grt import workloads
from helpers import mini

W = mini(workloads.C4, 12, (24, 16, 16))
BACK = workloads.C4_BACK_DISTANCE


def _forward(oracle, p, grid, m_abs, m_emis):
    ph = oracle.init_forward_photons(p, p.image_nx, p.image_ny, BACK)
    oracle.run(p, grid, ph, m_abs=m_abs, m_emis=m_emis)
    return oracle.image_products(p, ph).image_I


def test_oracle_gradient_matches_central_differences(oracle):
    p = W.params()
    grid = W.torus()
    shape = grid["r.npy"].shape
    ta, te = workloads.c4_target_multipliers(shape)
    target = _forward(oracle, p, grid, ta, te)
    m_abs = np.ones(shape)
    m_emis = np.ones(shape)
    img = _forward(oracle, p, grid, m_abs, m_emis)
    assert img.any() and not np.array_equal(img, target)
    dL = 2.0 * (img - target)
    ph = oracle.init_forward_photons(p, p.image_nx, p.image_ny, BACK)
    ga, ge = oracle.adjoint_image_I(p, grid, ph, dL, m_abs, m_emis)

    def loss(ma, me):
        return float(np.sum((_forward(oracle, p, grid, ma, me) - target) ** 2))

    rng = np.random.default_rng(7)
    h = 1e-6
    for g, which in ((ga, 0), (ge, 1)):
        nz = np.flatnonzero(np.abs(g) > 1e-3 * np.abs(g).max())
        assert nz.size > 0
        for cell in rng.choice(nz, size=min(6, nz.size), replace=False):
            ms = [m_abs.copy(), m_emis.copy()]
            ms[which].flat[cell] += h
            lp = loss(*ms)
            ms[which].flat[cell] -= 2 * h
            lm = loss(*ms)
            fd = (lp - lm) / (2 * h)
            assert abs(fd - g.flat[cell]) <= 1e-4 * abs(g.flat[cell]), (which, cell, fd, g.flat[cell])
    # cells no ray samples have zero gradient
    assert np.count_nonzero(ga) < ga.size and np.count_nonzero(ge) < ge.size
