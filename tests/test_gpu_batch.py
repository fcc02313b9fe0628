"""Batched images (grt_init_image_batch) and the render graph (grt_render_graph).

Every image of a batch runs the same per-ray arithmetic as that image traced
alone (its camera, frequency and coefficients come from the image table, ids
continue across images), so each image's photons and products must equal the
single-image run bit for bit, and the single-image run is the oracle's."""

import math

import numpy as np
import pytest

from grt import abi, workloads
from helpers import assert_photons_match, assert_products_match, mini, run_oracle, stokes_l2_rel

pytestmark = pytest.mark.gpu

SMALL = mini(workloads.C2, 16, (32, 16, 16))


def batch_specs(p):
    return [
        abi.ImageSpec.from_params(p, 16, 16, camera_theta=math.radians(17.0)),
        abi.ImageSpec.from_params(p, 12, 20, camera_theta=math.radians(60.0), custom_frequency_hz=86e9,
                                  emission_coefficient=86.0 / 230.0),
        abi.ImageSpec.from_params(p, 24, 24, camera_theta=math.radians(85.0), camera_phi=0.7,
                                  custom_frequency_hz=345e9, emission_coefficient=1.5, absorption_coefficient=0.5),
    ]


def single_params(p, sp):
    q = p.copy()
    q.update(camera_theta=sp.camera_theta, camera_phi=sp.camera_phi, camera_distance=sp.camera_distance,
             camera_width=sp.camera_width, camera_height=sp.camera_height, image_nx=sp.nx, image_ny=sp.ny,
             custom_frequency_hz=sp.custom_frequency_hz, absorption_coefficient=sp.absorption_coefficient,
             emission_coefficient=sp.emission_coefficient, nphotons=sp.nx * sp.ny)
    return q


def run_batch(lib, p, grid, specs, graph=False):
    ctx = lib.Context(p)
    try:
        ctx.upload_grid(grid)
        ctx.init_image_batch(specs)
        assert ctx.batch_image_count == len(specs)
        stats = ctx.render_graph() if graph else ctx.run()
        ph = ctx.download_photons()
        prods = [ctx.batch_image_products(k) for k in range(len(specs))]
    finally:
        ctx.close()
    return ph, prods, stats


def test_batch_equals_single_images(gpu, oracle):
    p = SMALL.params()
    grid = SMALL.torus()
    specs = batch_specs(p)
    ph, prods, stats = run_batch(gpu, p, grid, specs)
    start = 0
    accepted = 0
    for k, sp in enumerate(specs):
        q = single_params(p, sp)
        n = sp.nx * sp.ny
        ctx = gpu.Context(q)
        try:
            ctx.upload_grid(grid)
            ctx.init_image_photons(sp.nx, sp.ny, id_offset=start)
            st = ctx.run()
            single = ctx.download_photons()
            sprod = ctx.image_products()
        finally:
            ctx.close()
        accepted += st["accepted_steps"]
        for f in abi.PHOTON_FIELDS:
            assert np.array_equal(getattr(ph, f)[start:start + n], getattr(single, f)), (k, f)
        for f in ("image_I", "image_Q", "image_U", "image_V", "spectrum_frequency_hz", "arrived_count"):
            assert np.array_equal(getattr(prods[k], f), getattr(sprod, f)), (k, f)
        # spectrum bins sum many photons with atomics: equal up to summation order
        assert_products_match(prods[k], sprod)
        # and the single image is the oracle's
        init = oracle.init_image_photons(q, sp.nx, sp.ny, id_offset=start)
        want, wprod, _ = run_oracle(oracle, q, grid, photons=init)
        assert_photons_match(single, want)
        assert_products_match(sprod, wprod)
        start += n
    assert stats["accepted_steps"] == accepted
    assert stats["n_terminated"] == start


def test_render_graph_matches_run(gpu):
    p = SMALL.params()
    grid = SMALL.torus()
    specs = batch_specs(p)
    ph, prods, st = run_batch(gpu, p, grid, specs)
    ctx = gpu.Context(p)
    try:
        ctx.upload_grid(grid)
        ctx.init_image_batch(specs)
        for _ in range(3):  # capture, then replays from the re-initialised rays
            gst = ctx.render_graph()
            assert gst["accepted_steps"] == st["accepted_steps"]
            assert gst["steps_done"] == st["steps_done"]
            gph = ctx.download_photons()
            for f in abi.PHOTON_FIELDS:
                assert np.array_equal(getattr(gph, f), getattr(ph, f)), f
            for k in range(len(specs)):
                assert np.array_equal(ctx.batch_image_products(k).image_I, prods[k].image_I)
        # a parameter change re-captures: the replay equals a fresh run with
        # the new parameters (twice the energy per cell)
        q = p.copy()
        q.energy_per_cell_erg = 2.0 * p.energy_per_cell_erg
        ctx.set_params(q)
        ctx.init_image_batch(specs)
        ctx.render_graph()
        _, fresh, _ = run_batch(gpu, q, grid, specs)
        for k in range(len(specs)):
            assert_products_match(ctx.batch_image_products(k), fresh[k])
        assert not np.array_equal(fresh[0].image_I, prods[0].image_I)
    finally:
        ctx.close()


def test_render_graph_single_image(gpu):
    w = SMALL
    p = w.params()
    grid = w.torus()
    ctx = gpu.Context(p)
    try:
        ctx.upload_grid(grid)
        ctx.init_image_photons(w.pixels, w.pixels)
        st = ctx.run()
        want = ctx.image_products()
        ctx.init_image_photons(w.pixels, w.pixels)
        gst = ctx.render_graph()
        got = ctx.image_products()
        assert gst["accepted_steps"] == st["accepted_steps"]
        assert np.array_equal(got.image_I, want.image_I)
        # chunked runs cannot be captured
        q = p.copy()
        q.termination_percent = 0.5
        ctx.set_params(q)
        with pytest.raises(gpu.GrtError):
            ctx.render_graph()
    finally:
        ctx.close()


def test_batch_rejects_bad_specs(gpu):
    p = SMALL.params()
    ctx = gpu.Context(p)
    try:
        with pytest.raises(gpu.GrtError):
            ctx.init_image_batch([abi.ImageSpec.from_params(p, 0, 16)])
        with pytest.raises(gpu.GrtError):
            ctx.init_image_batch([abi.ImageSpec.from_params(p, 16, 16, camera_width=0.0)])
        with pytest.raises(gpu.GrtError):
            ctx.batch_image_products(0)
    finally:
        ctx.close()


@pytest.mark.parametrize("prec,bar", [(abi.PREC_MIXED, 1e-5), (abi.PREC_MIXED_GRID, 1e-3)],
                         ids=["mixed", "mixed_grid"])
def test_mixed_precision_batch_error(gpu, prec, bar):
    # each frequency channel of the C2 image (at 64x64 on a 64x32x32 grid) in
    # a mixed form against the FP64 form, L2 relative Stokes-I error: the
    # benchmark's 1e-5 bar for GRT_PREC_MIXED (FP32 only where the Stokes
    # vector no longer changes); GRT_PREC_MIXED_GRID, which also runs FP32
    # through the fluid after emission, is held to 1e-3 here and to the 1e-5
    # bar by the benchmark before it can be the headline form
    base = mini(workloads.C2, 64, (64, 32, 32))
    bw = workloads.BatchWorkload("c2_small_x4freq", base,
                                 [(base.inclination_deg, base.pixels, f) for f in workloads.FREQ_CHANNELS_GHZ])
    p = bw.params()
    grid = bw.torus()
    specs = bw.specs(p)
    _, ref, _ = run_batch(gpu, p, grid, specs)
    pm = p.copy()
    pm.precision = prec
    _, got, _ = run_batch(gpu, pm, grid, specs)
    for k in range(len(specs)):
        assert ref[k].image_I.any()
        err = stokes_l2_rel(got[k].image_I, ref[k].image_I)
        print(f"precision {prec} channel {k}: Stokes-I L2 relative error {err:.3g}")
        assert err <= bar, (k, err)


def channel_specs(p):
    # four frequency channels of one camera, plus one image with another camera
    f = [(230e9, 1.0), (345e9, 1.5), (86e9, 86.0 / 230.0), (43e9, 43.0 / 230.0)]
    specs = [abi.ImageSpec.from_params(p, 16, 16, camera_theta=math.radians(17.0), custom_frequency_hz=nu,
                                       emission_coefficient=j, absorption_coefficient=0.5 * j) for nu, j in f]
    specs.insert(2, abi.ImageSpec.from_params(p, 12, 12, camera_theta=math.radians(40.0)))
    return specs


@pytest.mark.parametrize("generator", [abi.GEN_CUSTOM, abi.GEN_BLACKBODY])
def test_channel_sharing_equals_single_images(gpu, oracle, generator):
    # The four channels share one geodesic per pixel; every channel must end
    # exactly as if traced alone (own id, draws, frequency and Stokes vector).
    w = mini(workloads.C2, 16, (32, 16, 16), generator=generator, temperature_k_per_code=1e10)
    p = w.params()
    grid = w.torus()
    specs = channel_specs(p)
    shared, sprods, sst = run_batch(gpu, p, grid, specs)
    ctx = gpu.Context(p)
    try:
        ctx.set_channel_sharing(False)
        ctx.upload_grid(grid)
        ctx.init_image_batch(specs)
        ust = ctx.run()
        unshared = ctx.download_photons()
    finally:
        ctx.close()
    for f in abi.PHOTON_FIELDS:
        assert np.array_equal(getattr(shared, f), getattr(unshared, f)), f
    n_shared_geodesics = 16 * 16 + 12 * 12
    assert sst["n_terminated"] == ust["n_terminated"] == shared.n
    assert sst["photon_calls"] < ust["photon_calls"]  # one geodesic per pixel for the four channels
    start = 0
    for k, sp in enumerate(specs):
        n = sp.nx * sp.ny
        q = single_params(p, sp)
        init = oracle.init_image_photons(q, sp.nx, sp.ny, id_offset=start)
        want, wprod, _ = run_oracle(oracle, q, grid, photons=init)
        got = abi.PhotonArrays.from_dict({f: getattr(shared, f)[start:start + n] for f in abi.PHOTON_FIELDS})
        assert_photons_match(got, want)
        assert_products_match(sprods[k], wprod)
        start += n
    assert n_shared_geodesics < shared.n


def test_all_batch_products_at_once(gpu):
    # grt_get_all_batch_image_products: the same products as one call per image
    p = SMALL.params()
    specs = batch_specs(p)
    ctx = gpu.Context(p)
    try:
        ctx.upload_grid(SMALL.torus())
        ctx.init_image_batch(specs)
        ctx.run()
        each = [ctx.batch_image_products(k) for k in range(len(specs))]
        outs = [abi.ProductArrays(sp.nx, sp.ny, p.spectrum_bins) for sp in specs]
        ctx.all_batch_image_products(outs)
        with pytest.raises(Exception, match="nimages"):
            ctx.all_batch_image_products(outs[:1])
    finally:
        ctx.close()
    for a, b in zip(outs, each):
        for f in ("image_I", "image_Q", "image_U", "image_V", "spectrum_frequency_hz", "spectrum_I", "arrived_count"):
            assert np.array_equal(getattr(a, f), getattr(b, f)), f
