"""Two-launch image mode (launch config split_legs = 1, the default): the
backward leg of every ray in one launch, the rest in a second launch over the
same queue.  Every photon takes the same calls in the same order as in one
launch over whole rays, so the final photon state, the image products and the
counters must equal the one-launch run bit for bit -- for both precision
forms, both integrators, batches whose frequency channels share a geodesic,
chunked termination (several launches per run), scattering and line-of-sight
forward rays."""

import math

import numpy as np
import pytest

from grt import abi, workloads
from helpers import mini

pytestmark = pytest.mark.gpu

C1_MINI = mini(workloads.C1, 16, (24, 16, 16))
C2_MINI = mini(workloads.C2, 24, (32, 16, 16))
STATS = ("accepted_steps", "rejected_attempts", "photon_calls", "n_terminated", "steps_done")


def trace(lib, p, grid, split, init, graph=False, sharing=True):
    ctx = lib.Context(p)
    try:
        ctx.set_launch_config(split_legs=int(split))
        ctx.set_channel_sharing(sharing)
        ctx.upload_grid(grid)
        init(ctx)
        st = ctx.render_graph() if graph else ctx.run()
        ph = ctx.download_photons()
        nimg = ctx.batch_image_count
        prods = [ctx.batch_image_products(k) for k in range(nimg)] if nimg else [ctx.image_products()]
    finally:
        ctx.close()
    return ph, prods, st


def assert_same(lib, p, grid, init, graph=False, sharing=True):
    a, pa, sa = trace(lib, p, grid, True, init, graph, sharing)
    b, pb, sb = trace(lib, p, grid, False, init, graph, sharing)
    for f in abi.PHOTON_FIELDS:
        assert np.array_equal(getattr(a, f), getattr(b, f)), f
    for x, y in zip(pa, pb):
        for f in ("image_I", "image_Q", "image_U", "image_V", "spectrum_I"):
            # atomics add in any order: equal within rounding, not bit for bit
            assert np.allclose(getattr(x, f), getattr(y, f), rtol=1e-12, atol=0.0), f
        assert int(x.arrived_count[0]) == int(y.arrived_count[0])
    for k in STATS:
        assert sa[k] == sb[k], (k, sa[k], sb[k])
    assert sa["launches"] == 3 * sb["launches"]  # backward leg, generation, the rest
    assert sa["timed_out"] == 0
    return a, sa


@pytest.mark.parametrize("precision", [abi.PREC_FP64, abi.PREC_MIXED], ids=["fp64", "mixed"])
@pytest.mark.parametrize("w", [C1_MINI, C2_MINI], ids=["c1_rk4", "c2_rk45"])
def test_split_equals_one_launch(gpu, w, precision):
    p = w.params()
    p.precision = precision
    ph, st = assert_same(gpu, p, w.torus(), lambda c: c.init_image_photons(w.pixels, w.pixels))
    assert (ph.phase == 3).sum() > 0 and st["n_terminated"] == ph.n


def channel_batch(p):
    specs = []
    for f in (230.0, 345.0, 86.0):
        specs.append(abi.ImageSpec.from_params(p, 16, 16, camera_theta=math.radians(17.0), custom_frequency_hz=f * 1e9,
                                               emission_coefficient=f / 230.0))
    specs.append(abi.ImageSpec.from_params(p, 12, 20, camera_theta=math.radians(60.0)))
    return specs


@pytest.mark.parametrize("graph", [False, True], ids=["run", "graph"])
@pytest.mark.parametrize("precision", [abi.PREC_FP64, abi.PREC_MIXED], ids=["fp64", "mixed"])
def test_split_batch_with_shared_channels(gpu, precision, graph):
    w = C2_MINI
    p = w.params()
    p.precision = precision
    specs = channel_batch(p)
    assert_same(gpu, p, w.torus(), lambda c: c.init_image_batch(specs), graph=graph)


@pytest.mark.parametrize("sharing", [True, False], ids=["shared", "unshared"])
def test_split_chunked_termination(gpu, sharing):
    # termination_percent < 1: the run is several chunks, each one (or two)
    # launches; photons still live at a chunk's end resume in the next chunk
    # in whichever leg they are in.
    w = mini(workloads.C2, 16, (32, 16, 16), termination_percent=0.9, output_interval=7,
             generator=abi.GEN_BLACKBODY, temperature_k_per_code=1e10)
    p = w.params()
    specs = channel_batch(p)
    ph, st = assert_same(gpu, p, w.torus(), lambda c: c.init_image_batch(specs), sharing=sharing)
    assert st["launches"] > 3 and st["steps_done"] < p.max_steps


def test_chunked_sharing_equals_unshared(gpu):
    # a shared geodesic resumes in the next chunk with the lead channel and
    # the finished channels the previous chunk left
    w = mini(workloads.C2, 16, (32, 16, 16), termination_percent=0.9, output_interval=5,
             generator=abi.GEN_BLACKBODY, temperature_k_per_code=1e10)
    p = w.params()
    specs = channel_batch(p)
    init = lambda c: c.init_image_batch(specs)  # noqa: E731
    for split in (True, False):
        a, _, sa = trace(gpu, p, w.torus(), split, init, sharing=True)
        b, _, sb = trace(gpu, p, w.torus(), split, init, sharing=False)
        for f in abi.PHOTON_FIELDS:
            assert np.array_equal(getattr(a, f), getattr(b, f)), (split, f)
        assert sa["n_terminated"] == sb["n_terminated"] and sa["steps_done"] == sb["steps_done"]


def test_split_with_scattering(gpu):
    w = mini(workloads.C2, 16, (32, 16, 16), scattering_enabled=1, scattering_albedo=0.8,
             density_g_cm3_per_code=0.5, length_cm_per_code=1.0)
    p = w.params()
    assert_same(gpu, p, w.torus(), lambda c: c.init_image_photons(w.pixels, w.pixels))


def test_split_forward_rays(gpu):
    # line-of-sight forward rays start in ImageForward: the backward-leg
    # launch has nothing to do and the second launch traces them whole
    w = workloads.scaled(workloads.C4, pixels=16, grid=(32, 16, 16))
    p = w.params()
    assert_same(gpu, p, w.torus(), lambda c: c.init_image_forward_photons(16, 16, workloads.C4_BACK_DISTANCE))
