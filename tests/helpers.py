"""Shared helpers for the parity tests: run a workload through the C ABI and
through the oracle on identical inputs, and compare."""

from __future__ import annotations

import numpy as np

import pyoracle
from grt import abi, workloads

FLOAT_FIELDS = ("frequency", "emission_frame_energy", "x0", "x1", "x2", "x3", "k0", "k1", "k2", "k3",
                "I", "Q", "U", "V", "dlambda", "theta_disp", "phi_disp")

# Parity tolerance of the FP64 form against the oracle (relative, per field).
FP64_RTOL = 1e-9


def mini(w, pixels, grid, **extra):
    return workloads.scaled(w, pixels=pixels, grid=grid, **extra)


def run_gpu(lib, p, grid, photons=None, nx=None, ny=None, launch=None):
    ctx = lib.Context(p)
    try:
        if launch:
            ctx.set_launch_config(**launch)
        ctx.upload_grid(grid)
        if photons is not None:
            ctx.upload_photons(photons)
        else:
            ctx.init_image_photons(nx, ny)
        stats = ctx.run()
        out = ctx.download_photons()
        prod = ctx.image_products()
    finally:
        ctx.close()
    return out, prod, stats


def run_oracle(oracle, p, grid, photons=None, nx=None, ny=None, m_abs=None, m_emis=None):
    ph = photons.copy() if photons is not None else oracle.init_image_photons(p, nx, ny)
    stats = oracle.run(p, grid, ph, m_abs=m_abs, m_emis=m_emis)
    prod = oracle.image_products(p, ph)
    return ph, prod, stats


def max_rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = np.maximum(np.maximum(np.abs(a), np.abs(b)), 1e-300)
    d = np.abs(a - b) / scale
    d[a == b] = 0.0
    return float(d.max()) if d.size else 0.0


def assert_photons_match(got, want, rtol=FP64_RTOL):
    d = pyoracle.compare_photons(got, want)
    assert d["id"] == 0 and d["terminate"] == 0 and d["phase"] == 0, d
    bad = {k: v for k, v in d.items() if k in FLOAT_FIELDS and v > rtol}
    assert not bad, bad
    return d


def assert_products_match(got, want, rtol=FP64_RTOL):
    assert int(got.arrived_count[0]) == int(want.arrived_count[0])
    for f in ("image_I", "image_Q", "image_U", "image_V", "spectrum_I", "spectrum_frequency_hz"):
        a, b = getattr(got, f), getattr(want, f)
        assert max_rel(a, b) <= rtol, (f, max_rel(a, b))


def stokes_l2_rel(a, b):
    """||a - b||_2 / ||b||_2 over an image."""
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / nb) if nb > 0 else float(np.linalg.norm(a - b))
