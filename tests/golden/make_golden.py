"""Generate the golden fixtures in this directory from the reference itself.

Run in a container where the reference tree is available (it is not on the
GPU box; the fixtures are committed instead):

    python tests/golden/make_golden.py --reference <reference project root>

(or GRT_REFERENCE_ROOT=<reference project root> in the environment)

Produces:
  torus_reference.npz  -- arrays written by the reference's own
      create_fishbone_moncrief_torus (src/create_example_data.py:102-281),
      imported with a stub matplotlib (only its plotting uses it), for two
      parameter sets; the product's torus generator must reproduce them bitwise.
  ref_run_<case>.npz   -- the reference's own integrate_geodesics
      (src/geodesic_integrate/integrate_cart_ks.hpp:423-535, compiled against
      oracle/shim by oracle/Makefile) on small image-mode cases: the
      pixel-grid initial photons, the final photon state (every field of
      struct Photons) and build_observation_products of the result.  Each
      case stores its parameters; the grid is rebuilt from them with the
      bitwise-checked torus generator.
  ref_known_answers.npz -- values of reference functions at fixed points:
      compute_hamiltonian_rhs, null_covariant_momentum_from_spatial_direction,
      geodesic observables, and locate_structured_grid_cell on the
      nonuniform 3x2x4 grid of src/tests/test_npy_loader.cpp.
"""

from __future__ import annotations

import argparse
import importlib.util
import os
import json
import sys
import tempfile
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT / "gr-ray-tracer_b200"))
sys.path.insert(0, str(ROOT / "oracle"))

TORUS_CASES = {
    "default": dict(nr=12, ntheta=8, nphi=6),
    "spin09": dict(nr=20, ntheta=10, nphi=8, spin=0.9, r_pressure_max=12.0, r_min=1.6),
}


def run_cases():
    from grt import abi, workloads
    return {
        "c1_rk4": workloads.scaled(workloads.C1, pixels=16, grid=(24, 16, 16)),
        "c2_rk45": workloads.scaled(workloads.C2, pixels=16, grid=(32, 16, 16)),
        "c2_rk45_chunked": workloads.scaled(workloads.C2, pixels=12, grid=(24, 12, 12), termination_percent=0.6,
                                            output_interval=3),
    }


def npy_loader_grid():
    """The nonuniform, fully 3-D 3x2x4 grid of src/tests/test_npy_loader.cpp:17-40."""
    r = np.zeros((3, 2, 4)); th = np.zeros((3, 2, 4)); ph = np.zeros((3, 2, 4))
    for i in range(3):
        for j in range(2):
            for k in range(4):
                r[i, j, k] = 1.0 + float(i * i) + 0.01 * j + 0.001 * k
                th[i, j, k] = 0.1 + 0.2 * float(j * j) + 0.005 * i
                ph[i, j, k] = 0.05 + 0.3 * float(k * k) + 0.002 * j
    return r, th, ph


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("GRT_REFERENCE_ROOT"))
    args = ap.parse_args()
    if not args.reference:
        ap.error("--reference (or GRT_REFERENCE_ROOT) must name the reference project's root")
    ref_src = Path(args.reference) / "src"

    # 1. torus arrays from the reference script
    mpl = types.ModuleType("matplotlib")
    mpl.rcParams = {}
    mpl.pyplot = types.ModuleType("matplotlib.pyplot")
    sys.modules["matplotlib"] = mpl
    sys.modules["matplotlib.pyplot"] = mpl.pyplot
    spec = importlib.util.spec_from_file_location("create_example_data", ref_src / "create_example_data.py")
    ced = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(ced)
    out = {}
    for name, kw in TORUS_CASES.items():
        with tempfile.TemporaryDirectory() as d:
            ced.create_fishbone_moncrief_torus(output_dir=d, plot=False, **kw)
            for f in ("r", "theta", "phi", "rho", "Tgas", "vel", "mag"):
                out[f"{name}/{f}"] = np.load(Path(d) / f"{f}.npy")
    out["cases"] = np.array(json.dumps(TORUS_CASES))
    np.savez_compressed(HERE / "torus_reference.npz", **out)

    # 2. reference runs
    import pyoracle
    from grt import abi, config, torus
    pyoracle.build(with_ref=True)
    ref = pyoracle.Reference()
    for name, w in run_cases().items():
        p = w.params()
        with tempfile.TemporaryDirectory() as d:
            d = Path(d)
            torus.write_numpy_dir(w.torus(), d / "np")
            toml = config.write_toml(p, d / "c.toml", d / "np", d / "out")
            init = ref.init_image_photons(toml, w.pixels, w.pixels)
            fin = init.copy()
            prod, st = ref.run(toml, fin, p)
        rec = {"params": np.array(json.dumps(p.as_dict())),
               "workload": np.array(json.dumps({"grid": list(w.grid), "spin": w.spin, "pixels": w.pixels})),
               "stepped": np.array(st["stepped"])}
        for f in abi.PHOTON_FIELDS:
            rec[f"init/{f}"] = getattr(init, f)
            rec[f"final/{f}"] = getattr(fin, f)
        for f, v in prod.as_dict().items():
            rec[f"products/{f}"] = v
        np.savez_compressed(HERE / f"ref_run_{name}.npz", **rec)

    # 3. known answers of reference functions
    ka = {}
    X = np.array([0.0, 5.0, -7.0, 2.0])
    K = np.array([0.4, -0.5, 0.768])
    for a in (1.0, 0.9, 0.94):
        ok, P = ref.null_momentum(X, K, a, 1.0)
        ka[f"a{a}/null_p"] = P
        ka[f"a{a}/rhs"] = ref.rhs(X, P, a, 1.0)
        ka[f"a{a}/observables"] = ref.observables(np.concatenate([X, P]), a, 1.0)
    ka["X"] = X
    ka["K"] = K
    r, th, ph = npy_loader_grid()
    ok, ijk = ref.locate_cell(r, th, ph, r[2, 1, 3], th[2, 1, 3], ph[2, 1, 3])
    ka["npy_loader/located"] = np.array([int(ok), *ijk])
    rng = np.random.default_rng(0)
    q = []
    for _ in range(200):
        i, j, k = rng.integers(0, 3), rng.integers(0, 2), rng.integers(0, 4)
        pt = (r[i, j, k] * np.exp(rng.normal(0, 0.2)), th[i, j, k] + rng.normal(0, 0.05),
              (ph[i, j, k] + rng.normal(0, 0.1)) % (2 * np.pi))
        ok, ijk = ref.locate_cell(r, th, ph, *pt)
        q.append([*pt, int(ok), *ijk])
    ka["npy_loader/random_queries"] = np.array(q)
    np.savez_compressed(HERE / "ref_known_answers.npz", **ka)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
