"""The allocation-free entry point, grt_trace_device_noalloc.

It exists for callers that cannot call cudaMalloc where they trace -- hosts
whose device memory belongs to their own pool or a fixed budget, and loops
that must not allocate after start-up because cudaMalloc can synchronise the
device.  Such a caller keeps the grid and the photons in device memory it
already owns; this entry point traces them in place, keeping its own scratch
(work-queue head, counters, staged grid axes) in a 128 KiB array inside the
library, so it allocates nothing.

Here the test (not the entry point) owns the device memory, through torch.
The results must match the ordinary context entry point (grt_upload_grid /
grt_upload_photons / grt_run) within the FP64 parity tolerance, on two calls
in a row: the shared scratch keeps the last call's contents, so the second
call proves the entry point clears what must start at zero.  This file is
named to be collected last.
"""

import ctypes as C

import numpy as np
import pytest

from grt import abi, workloads
from helpers import assert_photons_match, mini, run_gpu

pytestmark = pytest.mark.gpu


def _device_soa(torch, init):
    """Copy a host PhotonArrays to device tensors; return (tensors, PhotonSoA of device pointers)."""
    t = {}
    for f in abi.PHOTON_FIELDS:
        a = getattr(init, f)
        if f == "id":
            a = a.view(np.int64)
        t[f] = torch.from_numpy(np.ascontiguousarray(a).copy()).cuda()
    soa = abi.PhotonSoA()
    ptr = lambda x, ct: C.cast(C.c_void_p(x.data_ptr()), C.POINTER(ct))
    soa.id = ptr(t["id"], C.c_uint64)
    for f in abi.PHOTON_FIELDS[1:18]:
        setattr(soa, f, ptr(t[f], C.c_double))
    soa.terminate = ptr(t["terminate"], C.c_uint8)
    soa.phase = ptr(t["phase"], C.c_uint8)
    return t, soa


def _to_host(t, n):
    out = abi.PhotonArrays(n)
    for f in abi.PHOTON_FIELDS:
        a = t[f].cpu().numpy()
        setattr(out, f, a.view(np.uint64) if f == "id" else a)
    return out


@pytest.mark.parametrize("w", [mini(workloads.C2, 24, (32, 16, 16)), mini(workloads.C1, 12, (24, 16, 16))],
                         ids=["rk45", "rk4"])
def test_noalloc_matches_context_entry_point_twice(gpu, oracle, w):
    torch = pytest.importorskip("torch")
    p = w.params()
    grid = w.torus()
    init = oracle.init_image_photons(p, w.pixels, w.pixels)
    want, _, wst = run_gpu(gpu, p, grid, photons=init)

    dgrid = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in grid.items()}
    G = abi.DeviceGrid()
    G.nr, G.ntheta, G.nphi = grid["r.npy"].shape
    for field, key in (("r", "r.npy"), ("theta", "theta.npy"), ("phi", "phi.npy"), ("rho", "rho.npy"),
                       ("temperature", "Tgas.npy"), ("vel4", "vel.npy"), ("mag4", "mag.npy")):
        setattr(G, field, dgrid[key].data_ptr())
    for _ in range(2):
        tensors, soa = _device_soa(torch, init)
        torch.cuda.synchronize()
        st = gpu.trace_device_noalloc(p, G, soa, init.n)
        torch.cuda.synchronize()
        got = _to_host(tensors, init.n)
        assert_photons_match(got, want)
        for key in ("accepted_steps", "rejected_attempts", "photon_calls", "n_terminated", "steps_done"):
            assert st[key] == wst[key], key


def test_noalloc_rejects_oversized_grid(gpu):
    p = workloads.C2.params()
    G = abi.DeviceGrid()
    G.nr, G.ntheta, G.nphi = 8000, 100, 100
    with pytest.raises(gpu.GrtError, match="nr \\+ ntheta \\+ nphi must be <= 8160"):
        gpu.trace_device_noalloc(p, G, abi.PhotonSoA(), 0)
