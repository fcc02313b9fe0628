"""Host side of the multi-GPU paths, on CPU with the gloo backend (two ranks):
row sharding of one image, image sharding of a batch, and the product
reduction.  Each rank traces its rows with the oracle (the kernels need a
GPU); summing the ranks' products must give the single-process products."""

import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from grt import abi, parallel, workloads
from helpers import mini

W = mini(workloads.C1, 12, (24, 16, 16))


def test_row_range_covers_every_row_once():
    for ny in (1, 7, 64, 257):
        for world in (1, 2, 3, 8):
            rows = []
            for r in range(world):
                r0, n = parallel.row_range(ny, world, r)
                rows.extend(range(r0, r0 + n))
            assert rows == list(range(ny)), (ny, world)


def test_shard_images_balances_and_covers():
    costs = [64 * 64, 512 * 512, 128 * 128, 256 * 256, 64 * 64, 512 * 512, 256 * 256]
    shards = parallel.shard_images(costs, 3)
    assert sorted(i for s in shards for i in s) == list(range(len(costs)))
    loads = [sum(costs[i] for i in s) for s in shards]
    assert max(loads) - min(loads) <= max(costs)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parent.parent
    for p in (str(root / "gr-ray-tracer_b200"), str(root / "oracle"), str(root / "tests")):
        if p not in sys.path:
            sys.path.insert(0, p)
    import pyoracle
    from grt import parallel as par
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        o = pyoracle.Oracle()
        p = W.params()
        grid = W.torus()
        nx = ny = W.pixels
        full = o.init_image_photons(p, nx, ny)
        row0, nrows = par.row_range(ny, world, rank)
        lo, hi = row0 * nx, (row0 + nrows) * nx
        mine = abi.PhotonArrays.from_dict({f: getattr(full, f)[lo:hi].copy() for f in abi.PHOTON_FIELDS})
        o.run(p, grid, mine)
        prod = o.image_products(p, mine)
        par.reduce_products(prod, dst=0)
        if rank == 0:
            o.run(p, grid, full)
            want = o.image_products(p, full)
            np.savez(os.path.join(out_dir, "r.npz"), **{f"got_{k}": v for k, v in prod.as_dict().items()},
                     **{f"want_{k}": v for k, v in want.as_dict().items()})
        # replica path: every rank's whole image, summed on all ranks
        rep = o.image_products(p, mine)
        par.all_reduce_products(rep)
        np.save(os.path.join(out_dir, f"all_{rank}.npy"), rep.image_I)
    finally:
        dist.destroy_process_group()


def test_row_sharded_image_reduces_to_single_process(tmp_path):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    r = np.load(tmp_path / "r.npz")
    for k in ("image_I", "image_Q", "image_U", "image_V", "spectrum_I"):
        got, want = r[f"got_{k}"], r[f"want_{k}"]
        assert np.allclose(got, want, rtol=1e-12, atol=0.0), k
    assert int(r["got_arrived_count"][0]) == int(r["want_arrived_count"][0])
    assert r["want_image_I"].any()
    a0, a1 = np.load(tmp_path / "all_0.npy"), np.load(tmp_path / "all_1.npy")
    assert np.array_equal(a0, a1)
    assert np.allclose(a0, r["want_image_I"], rtol=1e-12, atol=0.0)


IMAGES = [15.0, 40.0, 60.0, 80.0, 30.0]  # inclinations of a small batch, one image each


def _images_rank_main(rank, world, port, out_dir):
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parent.parent
    for p in (str(root / "gr-ray-tracer_b200"), str(root / "oracle"), str(root / "tests")):
        if p not in sys.path:
            sys.path.insert(0, p)
    import math
    import pyoracle
    from grt import parallel as par
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        o = pyoracle.Oracle()
        grid = W.torus()
        shards = par.shard_images([W.pixels ** 2] * len(IMAGES), world)
        slots = max(len(sh) for sh in shards)

        def products_of(k):
            p = W.params()
            p.camera_theta = math.radians(IMAGES[k])
            ph = o.init_image_photons(p, W.pixels, W.pixels)
            o.run(p, grid, ph)
            return par._flat(o.image_products(p, ph))

        size = products_of(0).size
        block = np.zeros(slots * size)
        for j, k in enumerate(shards[rank]):
            block[j * size:(j + 1) * size] = products_of(k)
        parts = par.all_gather_blocks(block)
        if rank == 0:
            got = np.zeros((len(IMAGES), size))
            for r, sh in enumerate(shards):
                for j, k in enumerate(sh):
                    got[k] = parts[r][j * size:(j + 1) * size]
            want = np.stack([products_of(k) for k in range(len(IMAGES))])
            np.savez(os.path.join(out_dir, "images.npz"), got=got, want=want)
    finally:
        dist.destroy_process_group()


def test_sharded_images_gather_to_single_process(tmp_path):
    """Whole images assigned to two ranks by shard_images, each rank's
    products gathered on every rank: rank 0 reassembles every image equal to
    the single-process run."""
    world = 2
    mp.start_processes(_images_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    r = np.load(tmp_path / "images.npz")
    assert np.array_equal(r["got"], r["want"])
    assert (r["want"] != 0).any(axis=1).all()
