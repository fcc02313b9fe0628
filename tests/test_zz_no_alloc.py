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

import pyoracle
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


def _device_grid(torch, grid):
    dgrid = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in grid.items()}
    G = abi.DeviceGrid()
    G.nr, G.ntheta, G.nphi = grid["r.npy"].shape
    for field, key in (("r", "r.npy"), ("theta", "theta.npy"), ("phi", "phi.npy"), ("rho", "rho.npy"),
                       ("temperature", "Tgas.npy"), ("vel4", "vel.npy"), ("mag4", "mag.npy")):
        setattr(G, field, dgrid[key].data_ptr())
    return dgrid, G


def _twice_against_context(gpu, torch, p, grid, init, exact=False):
    """Trace init through the context entry point once and through the
    allocation-free one twice in a row; both allocation-free results must
    match the context's (bit for bit when exact), with the same counts."""
    want, _, wst = run_gpu(gpu, p, grid, photons=init)
    dgrid, G = _device_grid(torch, grid)
    for _ in range(2):
        tensors, soa = _device_soa(torch, init)
        torch.cuda.synchronize()
        st = gpu.trace_device_noalloc(p, G, soa, init.n)
        torch.cuda.synchronize()
        got = _to_host(tensors, init.n)
        d = assert_photons_match(got, want)
        if exact:
            assert all(v == 0 for v in d.values()), d
        for key in ("accepted_steps", "rejected_attempts", "photon_calls", "n_terminated", "steps_done"):
            assert st[key] == wst[key], key
    return want


@pytest.mark.parametrize("w", [mini(workloads.C2, 24, (32, 16, 16)), mini(workloads.C1, 12, (24, 16, 16))],
                         ids=["rk45", "rk4"])
def test_noalloc_matches_context_entry_point_twice(gpu, oracle, w):
    torch = pytest.importorskip("torch")
    p = w.params()
    _twice_against_context(gpu, torch, p, w.torus(), oracle.init_image_photons(p, w.pixels, w.pixels))


def test_noalloc_non_separable_grid(gpu, oracle):
    """Coordinates perturbed cell by cell, so the grid is not an outer product
    of axes: both entry points take the reference's general three-pass lookup
    on the raw coordinate arrays."""
    torch = pytest.importorskip("torch")
    w = mini(workloads.C2, 20, (32, 16, 16))
    p = w.params()
    grid = dict(w.torus())
    rng = np.random.default_rng(8)
    grid["r.npy"] = grid["r.npy"] * (1.0 + 1e-4 * rng.standard_normal(grid["r.npy"].shape))
    grid["theta.npy"] = grid["theta.npy"] + 1e-5 * rng.standard_normal(grid["theta.npy"].shape)
    want = _twice_against_context(gpu, torch, p, grid, oracle.init_image_photons(p, w.pixels, w.pixels), exact=True)
    assert (want.phase == 3).sum() > 20  # rays arrived through the fluid


def _disk_packets(gpu, p, grid):
    ctx = gpu.Context(p)
    try:
        ctx.upload_grid(grid)
        n = ctx.init_disk_photons()
        init = ctx.download_photons()
    finally:
        ctx.close()
    assert n > 500
    p.nphotons = n
    return init


def test_noalloc_disk_mode_without_scattering(gpu):
    """Disk-mode packets from every cell, RK45, absorption and emission:
    photon for photon the same as the context entry point."""
    torch = pytest.importorskip("torch")
    wd = workloads.DiskWorkload("disk_small", (32, 16, 16), 0.9, 6.0, max_steps=4000)
    p = wd.params()
    p.scattering_enabled = 0
    grid = wd.torus()
    init = _disk_packets(gpu, p, grid)
    want = _twice_against_context(gpu, torch, p, grid, init, exact=True)
    assert (want.I != init.I).any()


def test_noalloc_disk_mode_with_scattering(gpu):
    """With Thomson scattering on, the allocation-free entry point reads the
    reference's raw grid layout and turns each sample's spherical four-vectors
    Cartesian with the GPU's sin/cos, where the context entry point uses
    vectors precomputed with the host's; an ulp in the fluid frame changes a
    scattered direction, so packets agree with the context entry point's in
    distribution (escape fraction, escape energy and direction), and each of
    the two calls in a row gives the same packets."""
    torch = pytest.importorskip("torch")
    scipy_stats = pytest.importorskip("scipy.stats")
    wd = workloads.DiskWorkload("disk_small", (32, 16, 16), 0.9, 6.0, max_steps=4000)
    p = wd.params()
    grid = wd.torus()
    init = _disk_packets(gpu, p, grid)
    want, _, _ = run_gpu(gpu, p, grid, photons=init)
    dgrid, G = _device_grid(torch, grid)
    runs = []
    for _ in range(2):
        tensors, soa = _device_soa(torch, init)
        torch.cuda.synchronize()
        st = gpu.trace_device_noalloc(p, G, soa, init.n)
        torch.cuda.synchronize()
        runs.append(_to_host(tensors, init.n))
        assert st["n_terminated"] == init.n
    d = pyoracle.compare_photons(runs[0], runs[1])
    assert all(v == 0 for v in d.values()), d

    def escapes(ph):
        r = np.sqrt(ph.x1 ** 2 + ph.x2 ** 2 + ph.x3 ** 2)
        esc = (ph.phase == 4) & (r > p.r_term_max)
        return esc, -ph.k0[esc], ph.x3[esc] / r[esc]

    (e1, E1, c1), (e2, E2, c2) = escapes(runs[0]), escapes(want)
    n = init.n
    f1, f2 = e1.mean(), e2.mean()
    assert abs(f1 - f2) <= 4 * np.sqrt(f1 * (1 - f1) / n + f2 * (1 - f2) / n) + 1e-12, (f1, f2)
    assert scipy_stats.ks_2samp(E1, E2).pvalue > 0.01
    assert scipy_stats.ks_2samp(c1, c2).pvalue > 0.01


def test_noalloc_samples_at_radial_cell_edges(gpu):
    """Photons placed so that their first fluid sample lands within a few ulp
    of a radial acceptance boundary, log(r / r_i) = +-0.500001 * (largest log
    spacing next to r_i): both entry points derive that bound with the same
    host routine, so they accept and reject exactly the same samples."""
    torch = pytest.importorskip("torch")
    w = mini(workloads.C1, 8, (24, 16, 16), max_steps=2)
    p = w.params()
    grid = w.torus()
    ra = grid["r.npy"][:, 0, 0]
    nr = len(ra)
    # interior edges (where the nearest cell changes) and the grid's inner
    # and outer edges (where samples start to be rejected)
    edges = []
    for i in range(2, nr - 2, 3):
        h = 0.500001 * max(abs(np.log(ra[i] / ra[i - 1])), abs(np.log(ra[i + 1] / ra[i])))
        edges += [ra[i] * np.exp(h), ra[i] * np.exp(-h)]
    edges += [ra[0] * np.exp(-0.500001 * abs(np.log(ra[0] / ra[1]))),
              ra[nr - 1] * np.exp(0.500001 * abs(np.log(ra[nr - 1] / ra[nr - 2])))]
    rows = [edge * (1.0 + k * 2.0 ** -52) for edge in edges for k in range(-24, 25)]
    r = np.array(rows)
    n = r.size
    ph = abi.PhotonArrays(n)
    ph.id[:] = np.arange(n, dtype=np.uint64)
    # equatorial plane (theta = pi/2 is inside the torus), phi = 0:
    # x^2 + y^2 = r^2 + a^2 for a Kerr-Schild radius r
    ph.x1[:] = np.sqrt(r * r + p.spin * p.spin)
    # a tiny momentum moves the photon by ~1e-14 M per unit of affine
    # parameter, so the sample after a step of 1 stays within a few ulp of
    # the start, while the transfer path of the step (|dlambda| = 1) is not small
    ph.k0[:] = -1e-14
    ph.k3[:] = 1e-16
    ph.dlambda[:] = 1.0
    ph.frequency[:] = 2.3e11
    ph.emission_frame_energy[:] = 1.0
    ph.I[:] = 1.0
    ph.phase[:] = 2  # ImageForward: every step samples the fluid and applies transfer
    want = _twice_against_context(gpu, torch, p, grid, ph, exact=True)
    changed = want.I != 1.0
    assert 0 < changed.sum() < n  # some samples accepted, some rejected at the edges


def test_noalloc_rejects_oversized_grid(gpu):
    p = workloads.C2.params()
    G = abi.DeviceGrid()
    G.nr, G.ntheta, G.nphi = 8000, 100, 100
    with pytest.raises(gpu.GrtError, match="nr \\+ ntheta \\+ nphi must be <= 8160"):
        gpu.trace_device_noalloc(p, G, abi.PhotonSoA(), 0)
