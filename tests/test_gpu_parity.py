"""Parity of the sm_100a kernels (through the C ABI) with the CPU oracle on the
same seeded inputs: per-ray final state and image products.  FP64 form:
every float field within 1e-9 relative (bitwise for the RK4 trajectory, which
uses only IEEE-exact operations); integer fields exact."""

import math

import numpy as np
import pytest

from grt import abi, torus, workloads
from helpers import (FP64_RTOL, assert_photons_match, assert_products_match, max_rel, mini, run_gpu,
                     run_oracle, stokes_l2_rel)

pytestmark = pytest.mark.gpu

C1_MINI = mini(workloads.C1, 16, (24, 16, 16))
C2_MINI = mini(workloads.C2, 24, (32, 16, 16))


@pytest.mark.parametrize("w", [C1_MINI, C2_MINI], ids=["c1_rk4", "c2_rk45"])
def test_image_parity_fp64(gpu, oracle, w):
    p = w.params()
    grid = w.torus()
    got, gprod, gst = run_gpu(gpu, p, grid, nx=w.pixels, ny=w.pixels)
    want, wprod, wst = run_oracle(oracle, p, grid, nx=w.pixels, ny=w.pixels)
    assert_photons_match(got, want)
    assert_products_match(gprod, wprod)
    assert gst["accepted_steps"] == wst["accepted_steps"]
    assert gst["rejected_attempts"] == wst["rejected_attempts"]
    assert gst["photon_calls"] == wst["photon_calls"]
    assert gst["n_terminated"] == wst["n_terminated"]
    assert gst["steps_done"] == wst["steps_done"]
    if w.integrator == abi.RK4:
        for f in ("x0", "x1", "x2", "x3", "k0", "k1", "k2", "k3"):
            assert np.array_equal(getattr(got, f), getattr(want, f)), f


@pytest.mark.parametrize("launch", [
    dict(threads_per_block=128, blocks_per_sm=2, refill_threshold=1, photons_per_grab=32, split_legs=0),
    dict(threads_per_block=128, blocks_per_sm=3, refill_threshold=16, photons_per_grab=64),
    dict(threads_per_block=128, blocks_per_sm=4, refill_threshold=32, photons_per_grab=4096),
])
def test_launch_shapes_identical(gpu, oracle, launch):
    w = C2_MINI
    p = w.params()
    grid = w.torus()
    base, bprod, _ = run_gpu(gpu, p, grid, nx=w.pixels, ny=w.pixels)
    got, gprod, _ = run_gpu(gpu, p, grid, nx=w.pixels, ny=w.pixels, launch=launch)
    for f in ("x1", "x2", "x3", "k1", "I", "dlambda", "phase", "terminate"):
        assert np.array_equal(getattr(got, f), getattr(base, f)), (launch, f)
    assert np.array_equal(gprod.image_I, bprod.image_I)


def test_chunked_termination_matches_reference_loop(gpu, oracle):
    # termination_percent < 1 with a short output interval: the loop stops on
    # the first output step whose terminated fraction reaches the threshold.
    w = mini(workloads.C1, 12, (24, 16, 16), termination_percent=0.5, output_interval=37)
    p = w.params()
    grid = w.torus()
    got, _, gst = run_gpu(gpu, p, grid, nx=w.pixels, ny=w.pixels)
    want, _, wst = run_oracle(oracle, p, grid, nx=w.pixels, ny=w.pixels)
    assert_photons_match(got, want)
    assert gst["steps_done"] == wst["steps_done"]
    assert gst["n_terminated"] == wst["n_terminated"]
    assert gst["launches"] > 1


@pytest.mark.parametrize("generator", [abi.GEN_BLACKBODY, abi.GEN_POWER_LAW])
def test_random_generators_match_draw_for_draw(gpu, oracle, generator):
    w = mini(workloads.C2, 16, (32, 16, 16), generator=generator, temperature_k_per_code=1e10,
             power_law_slope=2.5, nu_min_hz=1e9, nu_max_hz=1e14)
    p = w.params()
    grid = w.torus()
    got, gprod, _ = run_gpu(gpu, p, grid, nx=w.pixels, ny=w.pixels)
    want, wprod, _ = run_oracle(oracle, p, grid, nx=w.pixels, ny=w.pixels)
    assert_photons_match(got, want)
    assert_products_match(gprod, wprod)


def test_nonseparable_grid_uses_general_lookup(gpu, oracle):
    # Perturb the coordinates so they depend on every index (like the
    # reference's test_npy_loader grid): the kernel must fall back to the
    # reference's three-pass coordinate descent and still agree.
    w = mini(workloads.C2, 12, (20, 12, 12))
    p = w.params()
    grid = w.torus()
    nr, nth, nph = grid["r.npy"].shape
    i, j, k = np.meshgrid(np.arange(nr), np.arange(nth), np.arange(nph), indexing="ij")
    grid["r.npy"] = grid["r.npy"] * (1.0 + 1e-3 * np.sin(j + 2.0 * k))
    grid["theta.npy"] = grid["theta.npy"] + 1e-3 * np.cos(i + k)
    got, gprod, _ = run_gpu(gpu, p, grid, nx=w.pixels, ny=w.pixels)
    want, wprod, _ = run_oracle(oracle, p, grid, nx=w.pixels, ny=w.pixels)
    assert_photons_match(got, want)
    assert_products_match(gprod, wprod)


def test_long_separable_axes_use_general_lookup(gpu, oracle):
    # nr + ntheta + nphi above the shared-memory budget for staged axes
    # (10,240 values): the kernel keeps the axes in global memory and runs the
    # general lookup, with the same results
    w = mini(workloads.C2, 6, (10300, 2, 2))
    p = w.params()
    grid = w.torus()
    got, gprod, _ = run_gpu(gpu, p, grid, nx=w.pixels, ny=w.pixels)
    want, wprod, _ = run_oracle(oracle, p, grid, nx=w.pixels, ny=w.pixels)
    assert_photons_match(got, want)
    assert_products_match(gprod, wprod)


def test_vacuum_grid(gpu, oracle):
    w = mini(workloads.C2, 8, (16, 8, 8))
    p = w.params()
    got, _, gst = run_gpu(gpu, p, None, nx=w.pixels, ny=w.pixels)
    empty = {k: np.zeros((0, 0, 0) if k not in ("vel.npy", "mag.npy") else (0, 0, 0, 4))
             for k in torus.FIELD_FILES}
    want, _, _ = run_oracle(oracle, p, empty, nx=w.pixels, ny=w.pixels)
    assert_photons_match(got, want)
    # no fluid: backward rays never generate and leave through r_max
    assert np.all(got.phase == abi.PHASE_REJECTED)


def test_pre_terminated_and_empty(gpu, oracle):
    w = C2_MINI
    p = w.params()
    grid = w.torus()
    ph = oracle.init_image_photons(p, 8, 8)
    ph.terminate[::3] = 1
    got, _, gst = run_gpu(gpu, p, grid, photons=ph)
    want, _, wst = run_oracle(oracle, p, grid, photons=ph)
    assert_photons_match(got, want)
    assert np.array_equal(got.x1[::3], ph.x1[::3])
    # zero photons
    empty = abi.PhotonArrays(0)
    got0, _, st0 = run_gpu(gpu, p, grid, photons=empty)
    assert got0.n == 0 and st0["accepted_steps"] == 0


@pytest.mark.parametrize("w", [C1_MINI, C2_MINI, mini(workloads.C2, 64, (64, 32, 32))],
                         ids=["c1_rk4", "c2_rk45", "c2_rk45_64px"])
def test_mixed_precision_image_error(gpu, oracle, w):
    # Stokes-I image of the mixed FP32/FP64 form against the FP64 form:
    # L2 relative error at most 1e-5 (the benchmark's acceptance bar).
    p = w.params()
    grid = w.torus()
    ref, rprod, _ = run_gpu(gpu, p, grid, nx=w.pixels, ny=w.pixels)
    pm = p.copy()
    pm.precision = abi.PREC_MIXED
    got, gprod, _ = run_gpu(gpu, pm, grid, nx=w.pixels, ny=w.pixels)
    err = stokes_l2_rel(gprod.image_I, rprod.image_I)
    assert err <= 1e-5, err


def test_host_photon_block_moves_in_one_copy(gpu):
    # a host SoA in the library's block layout (one transfer each way) and a
    # SoA of separate arrays (one transfer per field) carry the same photons
    w = C2_MINI
    p = w.params()
    grid = w.torus()
    outs = []
    for block in (True, False):
        ctx = gpu.Context(p)
        try:
            ctx.upload_grid(grid)
            ctx.init_image_photons(w.pixels, w.pixels)
            n = ctx.n
            host = abi.PhotonArrays.block(n) if block else abi.PhotonArrays(n)
            ctx.download_photons(host)
            host.terminate[::5] = 1
            ctx.upload_photons(host)
            ctx.run()
            out = abi.PhotonArrays.block(n) if block else abi.PhotonArrays(n)
            ctx.download_photons(out)
        finally:
            ctx.close()
        outs.append(out)
    for f in abi.PHOTON_FIELDS:
        assert np.array_equal(getattr(outs[0], f), getattr(outs[1], f)), f
    assert outs[0].terminate.all()
