"""Asynchronous renders of host photons (grt_render_async / grt_render_wait).

A render enqueues the photon upload, the trace, every image's products and
their copy back to the host, and returns at once.  Two contexts sharing one
stream and used in turn must give, render for render, the products and
statistics of the synchronous path (grt_upload_photons, grt_run,
grt_get_all_batch_image_products) on the same photons: images and counts bit
for bit, spectra up to the order of their atomic additions."""

import math

import numpy as np
import pytest

from grt import abi, workloads
from grt.lib import GrtError
from helpers import max_rel, mini

pytestmark = pytest.mark.gpu

SMALL = mini(workloads.C2, 16, (32, 16, 16))
FIELDS = ("image_I", "image_Q", "image_U", "image_V", "spectrum_frequency_hz", "spectrum_I", "arrived_count")
STATS = ("accepted_steps", "rejected_attempts", "photon_calls", "n_terminated", "steps_done", "launches")


def batch_specs(p):
    # three frequency channels of one camera (they share geodesics) and a
    # second camera on its own
    specs = [abi.ImageSpec.from_params(p, 16, 16, camera_theta=math.radians(17.0), custom_frequency_hz=f * 1e9,
                                       emission_coefficient=f / 230.0) for f in (230.0, 345.0, 86.0)]
    specs.append(abi.ImageSpec.from_params(p, 12, 20, camera_theta=math.radians(60.0)))
    return specs


def pinned_block(n):
    import torch
    t = torch.empty(146 * n, dtype=torch.uint8, pin_memory=True)
    pa = abi.PhotonArrays.block(n, t.numpy())
    pa._keep = t
    return pa


def new_outs(p, specs):
    return [abi.ProductArrays(sp.nx, sp.ny, p.spectrum_bins) for sp in specs]


def batch_context(lib, p, grid, specs, stream=None):
    ctx = lib.Context(p)
    if stream is not None:
        ctx.set_stream(stream)
    ctx.upload_grid(grid)
    ctx.init_image_batch(specs)
    return ctx


def two_inputs(lib, p, grid, specs):
    """The batch's initial photons, and the same photons with every initial
    step doubled (a different step sequence, so a different image)."""
    ctx = batch_context(lib, p, grid, specs)
    try:
        x = pinned_block(ctx.n)
        ctx.download_photons(x)
    finally:
        ctx.close()
    y = pinned_block(x.n)
    y._buffer[:] = x._buffer
    y.dlambda[:] *= 2.0
    return x, y


def sync_render(lib, p, grid, specs, photons):
    ctx = batch_context(lib, p, grid, specs)
    try:
        ctx.upload_photons(photons)
        st = ctx.run()
        outs = ctx.all_batch_image_products(new_outs(p, specs))
    finally:
        ctx.close()
    return outs, st


def test_async_renders_equal_sync_path(gpu):
    import torch
    p = SMALL.params()
    grid = SMALL.torus()
    specs = batch_specs(p)
    x, y = two_inputs(gpu, p, grid, specs)
    ref = {"x": sync_render(gpu, p, grid, specs, x), "y": sync_render(gpu, p, grid, specs, y)}
    assert not np.array_equal(ref["x"][0][0].image_I, ref["y"][0][0].image_I)
    assert ref["x"][0][0].arrived_count[0] > 0

    stream = torch.cuda.Stream()
    ctxs = [batch_context(gpu, p, grid, specs, stream.cuda_stream) for _ in range(2)]
    outs = [new_outs(p, specs) for _ in range(2)]
    inputs = {"x": x, "y": y}
    pending = [None, None]
    got = []

    def collect(c):
        st = ctxs[c].render_wait()
        got.append((pending[c], st, [{f: getattr(o, f).copy() for f in FIELDS} for o in outs[c]]))
        pending[c] = None

    try:
        for k, name in enumerate(["x", "y", "y", "x", "x", "y"]):
            c = k % 2
            if pending[c] is not None:
                collect(c)
            ctxs[c].render_async(inputs[name], outs[c])
            pending[c] = name
        for c in (0, 1):
            if pending[c] is not None:
                collect(c)
    finally:
        for ctx in ctxs:
            ctx.close()
    assert [g[0] for g in got] == ["x", "y", "y", "x", "x", "y"]
    for name, st, prods in got:
        ref_outs, ref_st = ref[name]
        for k, (a, b) in enumerate(zip(prods, ref_outs)):
            for f in FIELDS:
                if f == "spectrum_I":
                    # many rays per bin, summed by atomics: equal up to the order of the additions
                    assert max_rel(a[f], b.spectrum_I) <= 1e-12, (name, k, max_rel(a[f], b.spectrum_I))
                else:
                    # one ray per pixel and channel: bit for bit
                    assert np.array_equal(a[f], getattr(b, f)), (name, k, f)
        for key in STATS:
            assert st[key] == ref_st[key], (name, key)


def test_async_render_errors(gpu):
    p = SMALL.params()
    grid = SMALL.torus()
    specs = batch_specs(p)
    x, _ = two_inputs(gpu, p, grid, specs)
    ctx = batch_context(gpu, p, grid, specs)
    try:
        outs = new_outs(p, specs)
        with pytest.raises(GrtError) as e:
            ctx.render_wait()
        assert e.value.status == abi.GRT_ESTATE
        # separate field arrays are not a photon block
        with pytest.raises(GrtError) as e:
            ctx.render_async(x.copy(), outs)
        assert e.value.status == abi.GRT_EINVAL
        # a block of another photon count
        with pytest.raises(GrtError) as e:
            ctx.render_async(pinned_block(x.n - 1), outs)
        assert e.value.status == abi.GRT_EINVAL
        with pytest.raises(GrtError) as e:
            ctx.render_async(x, outs[:-1])
        assert e.value.status == abi.GRT_EINVAL
        ctx.render_async(x, outs)
        with pytest.raises(GrtError) as e:
            ctx.render_async(x, outs)
        assert e.value.status == abi.GRT_ESTATE
        # the render in flight owns the context's device buffers: other work is refused until the wait
        for call in (ctx.run, lambda: ctx.upload_photons(x), ctx.download_photons, ctx.render_graph,
                     lambda: ctx.batch_image_products(0), lambda: ctx.init_image_batch(specs)):
            with pytest.raises(GrtError) as e:
                call()
            assert e.value.status == abi.GRT_ESTATE
        st = ctx.render_wait()
        assert st["n_terminated"] == x.n
        # and accepted again after it
        ctx.upload_photons(x)
        assert ctx.run()["n_terminated"] == x.n
    finally:
        ctx.close()
    # a single image (grt_init_image_photons) is not a batch
    q = SMALL.params()
    ctx = gpu.Context(q)
    try:
        ctx.upload_grid(grid)
        ctx.init_image_photons(16, 16)
        ph = pinned_block(ctx.n)
        ctx.download_photons(ph)
        with pytest.raises(GrtError) as e:
            ctx.render_async(ph, [abi.ProductArrays(16, 16, q.spectrum_bins)])
        assert e.value.status == abi.GRT_ESTATE
    finally:
        ctx.close()
