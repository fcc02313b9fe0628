"""The synthetic-input generator against arrays the reference's own
create_fishbone_moncrief_torus wrote (tests/golden/torus_reference.npz,
made by tests/golden/make_golden.py): bitwise identical."""

import json

import numpy as np
import pytest

from conftest import GOLDEN
from grt import torus


@pytest.mark.parametrize("case", ["default", "spin09"])
def test_torus_bitwise_equals_reference_script(case):
    g = np.load(GOLDEN / "torus_reference.npz")
    kw = json.loads(str(g["cases"]))[case]
    mine = torus.fishbone_moncrief_torus(**kw)
    for f in ("r", "theta", "phi", "rho", "Tgas", "vel", "mag"):
        ref = g[f"{case}/{f}"]
        got = mine[f + ".npy"]
        assert got.shape == ref.shape, f
        assert np.array_equal(got.view(np.uint64), ref.view(np.uint64)), f


def test_benchmark_torus_parameters():
    a = torus.benchmark_torus(16, 8, 8, spin=0.9)
    r, th = a["r.npy"], a["theta.npy"]
    horizon = 1.0 + np.sqrt(1.0 - 0.81)
    assert np.isclose(r[0, 0, 0], 1.05 * horizon) and np.isclose(r[-1, 0, 0], 50.0)
    assert np.isclose(th[0, 0, 0], 0.01) and np.isclose(th[0, -1, 0], np.pi - 0.01)
    assert a["rho.npy"].min() == 1e-6 and a["rho.npy"].max() == 1.0


def test_numpy_dir_roundtrip(tmp_path):
    a = torus.fishbone_moncrief_torus(6, 4, 4)
    torus.write_numpy_dir(a, tmp_path)
    b = torus.load_numpy_dir(tmp_path)
    for k in torus.FIELD_FILES:
        assert np.array_equal(a[k], b[k])
    (tmp_path / "mag.npy").unlink()
    with pytest.raises(FileNotFoundError, match="missing required file"):
        torus.load_numpy_dir(tmp_path)


def test_generator_validation():
    with pytest.raises(ValueError):
        torus.fishbone_moncrief_torus(1, 4, 4)
    with pytest.raises(ValueError):
        torus.fishbone_moncrief_torus(4, 4, 4, spin=1.5)
    with pytest.raises(ValueError):
        torus.fishbone_moncrief_torus(4, 4, 4, r_in=12.0, r_pressure_max=6.0)
