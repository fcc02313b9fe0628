import os
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
PKG = ROOT / "gr-ray-tracer_b200"
for p in (str(PKG), str(ROOT / "oracle"), str(ROOT / "tests"), str(ROOT / "tests" / "golden")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (B200)")


def _ensure_built():
    lib = PKG / "lib" / "libgrt_b200.so"
    if not lib.exists():
        subprocess.run(["make", "-s", "-j", "4", "-C", str(PKG)], check=True)
    if not (ROOT / "oracle" / "liboracle.so").exists():
        subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "oracle"], check=True)


_ensure_built()


@pytest.fixture(scope="session")
def oracle():
    import pyoracle
    return pyoracle.Oracle()


@pytest.fixture(scope="session")
def reference():
    import pyoracle
    if not pyoracle.Reference.available():
        pytest.skip("oracle/_ref/libgrt_ref.so not built (reference tree absent at build time)")
    return pyoracle.Reference()


@pytest.fixture(scope="session")
def gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from grt import lib
    return lib
