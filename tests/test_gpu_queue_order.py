"""The trace queue's schedule decides only which lane traces which ray, never
what a ray computes.  Image-mode queues hand each warp an 8 x 4 tile of pixels
(cut at the screen's right and bottom edges), and when every claim of a launch
fits in the resident warps the first claims are spread over the SMs.  These
check that schedule on screens whose sides are not multiples of the tile:
each ray against the oracle, and a frequency-channel batch of such a screen
(tiles over the channel group's geodesics) against its images traced alone."""

import math

import numpy as np
import pytest

from grt import abi, workloads
from helpers import assert_photons_match, assert_products_match, mini, run_gpu, run_oracle

pytestmark = pytest.mark.gpu

C2_SMALL = mini(workloads.C2, 16, (32, 16, 16))


def screen_params(w, nx, ny):
    p = w.params()
    p.update(image_nx=nx, image_ny=ny, nphotons=nx * ny)
    return p


@pytest.mark.parametrize("nx,ny", [(13, 7), (9, 21), (1, 6), (37, 3)])
def test_cut_tiles_match_oracle(gpu, oracle, nx, ny):
    p = screen_params(C2_SMALL, nx, ny)
    grid = C2_SMALL.torus()
    got, gprod, gst = run_gpu(gpu, p, grid, nx=nx, ny=ny)
    want, wprod, wst = run_oracle(oracle, p, grid, nx=nx, ny=ny)
    assert_photons_match(got, want)
    assert_products_match(gprod, wprod)
    assert gst["accepted_steps"] == wst["accepted_steps"]
    assert gst["rejected_attempts"] == wst["rejected_attempts"]


def test_cut_tiles_of_a_channel_group(gpu):
    # two frequency channels of one 13 x 7 screen share their geodesics: the
    # tiles run over the group's 91 geodesics; each channel must equal that
    # image traced alone, bit for bit
    p = screen_params(C2_SMALL, 13, 7)
    grid = C2_SMALL.torus()
    specs = [abi.ImageSpec.from_params(p, 13, 7, camera_theta=math.radians(17.0)),
             abi.ImageSpec.from_params(p, 13, 7, camera_theta=math.radians(17.0), custom_frequency_hz=86e9,
                                       emission_coefficient=86.0 / 230.0)]
    ctx = gpu.Context(p)
    try:
        ctx.upload_grid(grid)
        ctx.init_image_batch(specs)
        ctx.run()
        batch = ctx.download_photons()
        assert ctx.geodesics == 91
    finally:
        ctx.close()
    start = 0
    for sp in specs:
        q = p.copy()
        q.update(camera_theta=sp.camera_theta, custom_frequency_hz=sp.custom_frequency_hz,
                 emission_coefficient=sp.emission_coefficient)
        c = gpu.Context(q)
        try:
            c.upload_grid(grid)
            c.init_image_photons(13, 7, id_offset=start)
            c.run()
            single = c.download_photons()
        finally:
            c.close()
        for f in abi.PHOTON_FIELDS:
            assert np.array_equal(getattr(batch, f)[start:start + 91], getattr(single, f)), f
        start += 91


def test_reinitialised_layouts_match_fresh_contexts(gpu):
    # one context through three image sets: a batch, a single odd screen, the
    # batch again (the tile orders are rebuilt, then reused for the same
    # layout); each run must equal the same image set on a fresh context
    p = screen_params(C2_SMALL, 13, 7)
    grid = C2_SMALL.torus()
    specs = [abi.ImageSpec.from_params(p, 16, 12, camera_theta=math.radians(30.0)),
             abi.ImageSpec.from_params(p, 9, 5, camera_theta=math.radians(60.0), custom_frequency_hz=86e9)]

    def fresh(kind):
        c = gpu.Context(p)
        try:
            c.upload_grid(grid)
            c.init_image_batch(specs) if kind == "batch" else c.init_image_photons(13, 7)
            c.run()
            return c.download_photons()
        finally:
            c.close()

    want = {kind: fresh(kind) for kind in ("batch", "single")}
    ctx = gpu.Context(p)
    try:
        ctx.upload_grid(grid)
        for kind in ("batch", "single", "batch"):
            ctx.init_image_batch(specs) if kind == "batch" else ctx.init_image_photons(13, 7)
            ctx.run()
            got = ctx.download_photons()
            for f in abi.PHOTON_FIELDS:
                assert np.array_equal(getattr(got, f), getattr(want[kind], f)), (kind, f)
    finally:
        ctx.close()
