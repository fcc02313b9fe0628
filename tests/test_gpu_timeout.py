"""The trace kernels' give-up path.  A trace launch counts its warps' loop
iterations and stops past grt_launch_config.max_iterations: every lane
writes its photon back at its last call boundary (an RK45 call interrupted
between attempts is undone, so it reruns whole), the run returns
GRT_ETIMEOUT with stats.timed_out = 1, and the context stays usable.  The
limit is made to run out here by setting it small -- no fault, trap or
endless loop is involved -- and a second grt_run with the automatic limit
continues the photons to the same end state as one uninterrupted run."""

import ctypes as C

import numpy as np
import pytest

import pyoracle
from grt import abi, workloads
from helpers import FP64_RTOL, max_rel, mini, run_gpu

pytestmark = pytest.mark.gpu


def raw_run(ctx):
    st = abi.RunStats()
    rc = ctx.lib.grt_run(ctx.handle, C.byref(st))
    return rc, st.as_dict()


@pytest.mark.parametrize("split", [1, 0], ids=["split_legs", "one_launch"])
@pytest.mark.parametrize("form", ["rk45", "rk4"])
def test_iteration_limit_runs_out_and_the_run_resumes(gpu, split, form):
    base = workloads.C2 if form == "rk45" else workloads.C1
    w = mini(base, 24, (32, 16, 16))
    p = w.params()
    grid = w.torus()
    full, fprod, fst = run_gpu(gpu, p, grid, nx=24, ny=24, launch=dict(split_legs=split))
    assert fst["timed_out"] == 0 and fst["n_terminated"] == full.n
    ctx = gpu.Context(p)
    try:
        ctx.set_launch_config(split_legs=split, max_iterations=20)
        ctx.upload_grid(grid)
        ctx.init_image_photons(24, 24)
        rc, st = raw_run(ctx)
        assert rc == abi.GRT_ETIMEOUT
        assert st["timed_out"] == 1
        assert "iteration limit" in ctx.lib.grt_last_error(ctx.handle).decode()
        part = ctx.download_photons()
        live = part.terminate == 0
        assert live.any(), "the limit did not run out"
        assert st["n_terminated"] == int((~live).sum())
        # written back consistently: live photons hold finite state in a live
        # phase; photons that finished before the limit hold their final state
        for f in ("x0", "x1", "x2", "x3", "k0", "k1", "k2", "k3", "dlambda", "I"):
            assert np.isfinite(getattr(part, f)[live]).all(), f
        assert np.isin(part.phase[live], (1, 2)).all()
        for f in abi.PHOTON_FIELDS:
            assert np.array_equal(getattr(part, f)[~live], getattr(full, f)[~live]), f
        # the context is still usable: resume with the automatic limit
        ctx.set_launch_config(max_iterations=0)
        st2 = ctx.run()
        assert st2["timed_out"] == 0 and st2["n_terminated"] == full.n
        out = ctx.download_photons()
        prod = ctx.image_products()
    finally:
        ctx.close()
    d = pyoracle.compare_photons(out, full)
    assert all(v == 0 for v in d.values()), d
    assert int(prod.arrived_count[0]) == int(fprod.arrived_count[0])
    for f in ("image_I", "image_Q", "image_U", "image_V", "spectrum_I"):
        assert max_rel(getattr(prod, f), getattr(fprod, f)) <= (FP64_RTOL if f == "spectrum_I" else 1e-12), f


def test_negative_iteration_limit_is_rejected(gpu):
    ctx = gpu.Context(mini(workloads.C1, 8, (16, 8, 8)).params())
    try:
        with pytest.raises(gpu.GrtError, match="max_iterations"):
            ctx.set_launch_config(max_iterations=-1)
        assert ctx.launch_config()["max_iterations"] == 0
    finally:
        ctx.close()
