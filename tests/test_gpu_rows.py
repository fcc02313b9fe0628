"""One image split by pixel rows (grt_init_image_rows), as the ranks of a
multi-GPU render would trace it, on one GPU: each row range's rays equal
the corresponding rays of the whole image, and the products of the parts sum
to the whole image's products."""

import numpy as np
import pytest

from grt import abi, parallel, workloads
from helpers import assert_products_match, mini

pytestmark = pytest.mark.gpu

W = mini(workloads.C2, 24, (32, 16, 16))


def test_row_shards_sum_to_the_whole_image(gpu):
    p = W.params()
    grid = W.torus()
    nx = ny = W.pixels
    ctx = gpu.Context(p)
    try:
        ctx.upload_grid(grid)
        ctx.init_image_photons(nx, ny)
        ctx.run()
        whole = ctx.download_photons()
        want = ctx.image_products()
        world = 3
        total = None
        for r in range(world):
            row0, nrows = parallel.row_range(ny, world, r)
            ctx.init_image_rows(nx, ny, row0, nrows)
            ctx.run()
            part = ctx.download_photons()
            lo, hi = row0 * nx, (row0 + nrows) * nx
            for f in abi.PHOTON_FIELDS:
                assert np.array_equal(getattr(part, f), getattr(whole, f)[lo:hi]), (r, f)
            prod = ctx.image_products()
            if total is None:
                total = prod
            else:
                for f in ("image_I", "image_Q", "image_U", "image_V", "spectrum_I", "arrived_count"):
                    getattr(total, f)[...] += getattr(prod, f)
        total.spectrum_frequency_hz[...] = want.spectrum_frequency_hz
        assert_products_match(total, want)
        with pytest.raises(gpu.GrtError):
            ctx.init_image_rows(nx, ny, ny - 1, 2)
    finally:
        ctx.close()
