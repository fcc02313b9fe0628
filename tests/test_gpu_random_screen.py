"""The random-screen image initialisation on the GPU
(grt_init_image_photons_random): the rays equal the oracle's bit for bit
(same Philox streams keyed by 12345 + rank and photon id), and so does every
ray's trace and the image binned from them."""

import numpy as np
import pytest

import pyoracle
from grt import workloads
from helpers import FP64_RTOL, max_rel, mini

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("rank", [0, 3])
def test_random_screen_rays_and_trace_match_oracle(gpu, oracle, rank):
    w = mini(workloads.C2, 16, (32, 16, 16), rank=rank)
    p = w.params()
    grid = w.torus()
    n = 3000
    ctx = gpu.Context(p)
    try:
        ctx.upload_grid(grid)
        ctx.init_image_photons_random(n, id_offset=11)
        init = ctx.download_photons()
        st = ctx.run()
        out = ctx.download_photons()
        prod = ctx.image_products()
    finally:
        ctx.close()
    want = oracle.init_image_photons_random(p, n, id_offset=11)
    d = pyoracle.compare_photons(init, want)
    assert all(v == 0 for v in d.values()), d
    oracle.run(p, grid, want)
    d = pyoracle.compare_photons(out, want)
    assert all(v == 0 for v in d.values()), d
    assert st["n_terminated"] == n
    ref_prod = oracle.image_products(p, want)
    assert int(prod.arrived_count[0]) == int(ref_prod.arrived_count[0]) > 0
    assert prod.image_I.shape == (p.image_ny, p.image_nx)
    for f in ("image_I", "image_Q", "image_U", "image_V", "spectrum_I"):
        assert max_rel(getattr(prod, f), getattr(ref_prod, f)) <= (FP64_RTOL if f == "spectrum_I" else 1e-12), f
    if rank:
        # another rank draws other screen positions
        other = oracle.init_image_photons_random(mini(workloads.C2, 16, (32, 16, 16)).params(), n, id_offset=11)
        assert not np.array_equal(other.theta_disp, init.theta_disp)
