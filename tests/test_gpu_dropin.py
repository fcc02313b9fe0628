"""The drop-in through the reference's own executable.  oracle/Makefile
builds the reference's src/main.cpp twice against oracle/shim: unmodified
(oracle/_ref/gr-ray-trace) and with its integrate_geodesics call routed to
integrate_geodesics_b200 from include/grt_reference_adapter.hpp, linking
libgrt_b200.so (oracle/_ref/gr-ray-trace-b200).  Both read the same TOML
with the reference's own loader, initialise the same photons with the
reference's own initialize_photons_image, and write their archives with the
same names: every output-step archive must be byte for byte the reference's
(RK4 and RK45 trajectories are bit-identical), and the image products equal
per pixel (device atomics add a pixel's arrivals in another order)."""

import subprocess
from pathlib import Path

import numpy as np
import pytest

from grt import config, torus, workloads
from helpers import max_rel, mini

pytestmark = pytest.mark.gpu

REF_DIR = Path(__file__).resolve().parent.parent / "oracle" / "_ref"


def run_main(exe, toml, cwd):
    r = subprocess.run([str(exe), str(toml)], cwd=cwd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, (exe.name, r.returncode, r.stdout[-2000:], r.stderr[-2000:])


@pytest.mark.parametrize("form", ["rk4", "rk45"])
def test_reference_main_with_the_drop_in_writes_the_references_archives(gpu, form, tmp_path):
    plain, b200 = REF_DIR / "gr-ray-trace", REF_DIR / "gr-ray-trace-b200"
    if not (plain.exists() and b200.exists()):
        pytest.skip("oracle/_ref executables not built (reference tree absent at build time)")
    if form == "rk4":
        w = mini(workloads.C1, 16, (24, 16, 16), termination_percent=0.95, output_interval=50)
    else:
        w = mini(workloads.C2, 16, (32, 16, 16), termination_percent=0.95, output_interval=7)
    p = w.params()
    p.nphotons = 600  # the reference draws its own random screen positions
    torus.write_numpy_dir(w.torus(), tmp_path / "np")
    outs = {}
    for name, exe in (("ref", plain), ("b200", b200)):
        out = tmp_path / f"out_{name}"
        toml = config.write_toml(p, tmp_path / f"{name}.toml", tmp_path / "np", out)
        run_main(exe, toml, tmp_path)
        outs[name] = out
    ref_files = sorted(f.name for f in outs["ref"].iterdir())
    assert ref_files == sorted(f.name for f in outs["b200"].iterdir())
    steps = [f for f in ref_files if "_step_" in f]
    assert len(steps) >= 2
    for f in steps:
        assert (outs["b200"] / f).read_bytes() == (outs["ref"] / f).read_bytes(), f
    prod = [f for f in ref_files if f.endswith("_image_products.npz")]
    assert len(prod) == 1
    a, b = np.load(outs["b200"] / prod[0]), np.load(outs["ref"] / prod[0])
    assert list(a.keys()) == list(b.keys())
    assert int(a["arrived_count"][0]) == int(b["arrived_count"][0]) > 0
    for k in b.keys():
        assert a[k].dtype == b[k].dtype and a[k].shape == b[k].shape, k
        assert max_rel(a[k], b[k]) <= 1e-12, k
