"""Multi-GPU plumbing: one process per GPU, torch.distributed for the host side.

The hot path shards without any exchange: every ray is independent once the
grid (<= 55 MB) is replicated on each GPU.  The reference's MPI photon
exchange (photon_exchange.hpp) exists only because its ranks own grid slabs.
Two ways to use N GPUs:

* whole images: each rank traces its own images (shard_images assigns
  whole images to ranks, balancing rays); the only communication is gathering
  the products (all_gather_blocks; bench.py --gpus N renders one frame of a
  camera orbit per GPU and all-gathers the frames' products every step);
* one image split by pixel rows: row_range gives rank r its rows
  (grt_init_image_rows), every rank bins its arrivals into the full image and
  reduce_products sums the products over the ranks -- the analogue of the
  reference's product reduction (write_output.hpp:116-127).

Both collectives run once per render on small arrays (4*nx*ny + bins + 1
values), so NCCL's reduce (or gloo's on CPU) is the right tool; nothing on the
data path waits on another rank.
"""

from __future__ import annotations

import numpy as np


def row_range(ny: int, world: int, rank: int) -> tuple[int, int]:
    """Contiguous pixel rows (row0, nrows) of rank `rank` out of `world`;
    the first ny % world ranks take one extra row."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("need 0 <= rank < world")
    base, extra = divmod(int(ny), int(world))
    row0 = rank * base + min(rank, extra)
    return row0, base + (1 if rank < extra else 0)


def shard_images(costs, world: int) -> list[list[int]]:
    """Assign images (by index) to `world` ranks, longest-processing-time
    first: each image goes to the currently least-loaded rank.  `costs` are
    the images' estimated costs (e.g. pixel counts)."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    out = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += costs[i]
    return [sorted(x) for x in out]


def _flat(prod) -> np.ndarray:
    return np.concatenate([prod.image_I.ravel(), prod.image_Q.ravel(), prod.image_U.ravel(), prod.image_V.ravel(),
                           prod.spectrum_I.ravel(), prod.arrived_count.astype(np.float64).ravel()])


def reduce_products(prod, dst: int = 0, group=None):
    """Sum image products over the ranks of `group` onto rank `dst` (in place
    there; other ranks' buffers are left as they were).  Uses the process
    group's backend (NCCL on GPUs, gloo on CPU); on NCCL the flat buffer is
    staged through the current CUDA device."""
    import torch
    import torch.distributed as dist
    flat = _flat(prod)
    backend = dist.get_backend(group)
    t = torch.from_numpy(flat)
    if backend == "nccl":
        t = t.cuda()
    dist.reduce(t, dst=dst, op=dist.ReduceOp.SUM, group=group)
    if dist.get_rank(group) == dst:
        _unflat(prod, t.cpu().numpy())
    return prod


def all_reduce_products(prod, group=None):
    """Sum image products over the ranks of `group`, result on every rank."""
    import torch
    import torch.distributed as dist
    t = torch.from_numpy(_flat(prod))
    if dist.get_backend(group) == "nccl":
        t = t.cuda()
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    _unflat(prod, t.cpu().numpy())
    return prod


def _unflat(prod, flat: np.ndarray):
    n = prod.image_I.size
    o = 0
    for f in ("image_I", "image_Q", "image_U", "image_V"):
        getattr(prod, f)[...] = flat[o:o + n].reshape(getattr(prod, f).shape)
        o += n
    b = prod.spectrum_I.size
    prod.spectrum_I[...] = flat[o:o + b]
    o += b
    prod.arrived_count[...] = np.round(flat[o:o + 1]).astype(np.uint64)


def all_gather_blocks(block, group=None) -> list:
    """Every rank's block of equal size, in rank order, on every rank: the
    gather of image products when whole images are owned by single ranks.
    `block` is a 1-D numpy array or torch tensor; on NCCL it is staged
    through the current CUDA device.  Returns numpy arrays."""
    import numpy as np
    import torch
    import torch.distributed as dist
    t = block if isinstance(block, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(block))
    if dist.get_backend(group) == "nccl":
        t = t.cuda()
    parts = [torch.empty_like(t) for _ in range(dist.get_world_size(group))]
    dist.all_gather(parts, t, group=group)
    return [x.cpu().numpy() for x in parts]
