"""grt_copy_products_block: every image's products of the current image set
as one block in caller memory -- device memory for a collective, or host
memory -- in the documented layout, equal to what the per-image product calls
return."""

import numpy as np
import pytest

from grt import workloads
from helpers import mini

pytestmark = pytest.mark.gpu


def split_block(raw: np.ndarray, shapes, bins):
    f64 = raw.view(np.float64)
    out, o = [], 0
    for ny, nx in shapes:
        n = ny * nx
        out.append([f64[o + q * n:o + (q + 1) * n].reshape(ny, nx) for q in range(4)])
        o += 4 * n
    spectra = [f64[o + k * bins:o + (k + 1) * bins] for k in range(len(shapes))]
    o += len(shapes) * bins
    arrived = raw.view(np.uint64)[o:o + len(shapes)]
    return out, spectra, arrived


@pytest.mark.parametrize("where", ["device", "host"])
def test_products_block_equals_per_image_products(gpu, where):
    torch = pytest.importorskip("torch")
    base = mini(workloads.C2, 12, (32, 16, 16))
    bw = workloads.BatchWorkload("blk", base, [(17.0, 12, 230.0), (40.0, 16, 345.0), (60.0, 8, 86.0)])
    p = bw.params()
    ctx = gpu.Context(p)
    try:
        ctx.upload_grid(base.torus())
        ctx.init_image_batch(bw.specs())
        ctx.render_graph()
        nbytes = ctx.products_block_bytes
        want = [ctx.batch_image_products(k) for k in range(3)]
        if where == "device":
            buf = torch.zeros(nbytes, dtype=torch.uint8, device="cuda")
            ctx.copy_products_block(buf.data_ptr(), nbytes)
            ctx.synchronize()
            raw = buf.cpu().numpy()
        else:
            raw = np.zeros(nbytes, dtype=np.uint8)
            ctx.copy_products_block(raw.ctypes.data, nbytes)
            ctx.synchronize()
        with pytest.raises(gpu.GrtError, match="smaller than grt_products_block_bytes"):
            ctx.copy_products_block(raw.ctypes.data, nbytes - 8)
    finally:
        ctx.close()
    assert nbytes == 8 * sum(4 * px * px + p.spectrum_bins + 1 for _, px, _ in bw.images)
    images, spectra, arrived = split_block(raw, [(px, px) for _, px, _ in bw.images], p.spectrum_bins)
    for k in range(3):
        for q, f in enumerate(("image_I", "image_Q", "image_U", "image_V")):
            assert np.array_equal(images[k][q], getattr(want[k], f)), (k, f)
        assert np.array_equal(spectra[k], want[k].spectrum_I)
        assert int(arrived[k]) == int(want[k].arrived_count[0])
    assert arrived.sum() > 0
