"""The C ABI boundary without a GPU: the library loads, exports every
function include/grt.h declares, its structs have the ctypes layout, and the
TOML mirror parses configs exactly like the reference's own loader."""

import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

import pyoracle

from conftest import ROOT
from grt import abi, config, lib, workloads

HEADER = ROOT / "include" / "grt.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(grt_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_function():
    L = lib.load()
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert L.grt_abi_version() == 5


def test_struct_layout_matches_c(tmp_path):
    src = tmp_path / "sizes.c"
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "grt.h"', 'int main(void){']
    for cname, pyname in (("grt_params", abi.Params), ("grt_photon_soa", abi.PhotonSoA),
                          ("grt_run_stats", abi.RunStats), ("grt_image_products", abi.ImageProducts),
                          ("grt_launch_config", abi.LaunchConfig), ("grt_device_grid", abi.DeviceGrid),
                          ("grt_image_spec", abi.ImageSpec)):
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for f, _ in pyname._fields_:
            lines.append(f'printf("{cname}.{f} %zu\\n", offsetof({cname}, {f}));')
    lines.append("return 0;}")
    src.write_text("\n".join(lines))
    exe = tmp_path / "sizes"
    subprocess.run(["gcc", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    out = dict(line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split("\n") if line)
    for cname, pyname in (("grt_params", abi.Params), ("grt_photon_soa", abi.PhotonSoA),
                          ("grt_run_stats", abi.RunStats), ("grt_image_products", abi.ImageProducts),
                          ("grt_launch_config", abi.LaunchConfig), ("grt_device_grid", abi.DeviceGrid),
                          ("grt_image_spec", abi.ImageSpec)):
        assert int(out[cname]) == C.sizeof(pyname), cname
        for f, _ in pyname._fields_:
            assert int(out[f"{cname}.{f}"]) == getattr(pyname, f).offset, f"{cname}.{f}"


def test_defaults_are_the_reference_defaults():
    p = lib.default_params()
    r = config.reference_defaults()
    assert p.as_dict() == r.as_dict()


def _toml_cases():
    return {
        "c1": workloads.C1.params(),
        "c2": workloads.C2.params(),
        "disk": workloads.C2.params().update(mode=abi.MODE_DISK, scattering_enabled=1, generator=abi.GEN_BLACKBODY),
    }


@pytest.mark.parametrize("case", ["c1", "c2", "disk"])
def test_toml_mirror_matches_reference_loader(reference, tmp_path, case):
    p = _toml_cases()[case]
    t = config.write_toml(p, tmp_path / "c.toml", tmp_path / "np", tmp_path / "out", name="run")
    mine, npdir, outdir, name = lib.params_from_toml(t)
    ref = reference.params_from_toml(t)
    for k, v in ref.as_dict().items():
        if k in ("precision", "rank"):
            continue
        assert getattr(mine, k) == v, k
    assert npdir == str(tmp_path / "np") and outdir == str(tmp_path / "out") and name == "run"


def test_toml_mirror_on_reference_example_configs(reference):
    root = pyoracle.Reference.root()
    cfgs = sorted((root / "config").glob("*.toml")) if root else []
    if not cfgs:
        pytest.skip("the reference tree oracle/_ref was built from is not on this machine")
    for t in cfgs:
        mine, *_ = lib.params_from_toml(t)
        ref = reference.params_from_toml(t)
        for k, v in ref.as_dict().items():
            if k in ("precision", "rank"):
                continue
            assert getattr(mine, k) == v, (t.name, k)


@pytest.mark.parametrize("body,msg", [
    ("[black_hole]\nspin = 2.0\nmass = 1.0\n", "black_hole.spin must satisfy"),
    ("[integration]\nintegrator = \"euler\"\n", "integration.integrator must be"),
    ("[integration]\ntermination_percent = 1.5\n", "termination_percent must be in (0, 1]"),
    ("[photons]\ngenerator = \"laser\"\n", "photons.generator must be"),
    ("[scattering]\nenabled = yes\n", "scattering.enabled must be true or false"),
    ("[output]\ninterval = -3\n", "output.interval must not be negative"),
    ("this line is not a key value pair\n", "Malformed config line"),
])
def test_toml_errors_like_reference(tmp_path, body, msg):
    t = tmp_path / "bad.toml"
    t.write_text(body)
    with pytest.raises(lib.GrtError, match=re.escape(msg)):
        lib.params_from_toml(t)


def test_missing_config_file(tmp_path):
    with pytest.raises(lib.GrtError, match="Failed to open config file"):
        lib.params_from_toml(tmp_path / "nope.toml")


def test_param_validation():
    p = workloads.C2.params()
    lib.validate_params(p)
    p.camera_distance = -1.0
    with pytest.raises(lib.GrtError, match="camera distance"):
        lib.validate_params(p)


def test_host_photon_block_layout_matches_the_library():
    """abi.PhotonArrays.block lays the 20 fields out exactly where
    grt_host_photon_layout points them (the layout that moves in one copy)."""
    import ctypes as C

    import numpy as np

    from grt import abi, lib
    L = lib.load()
    for n in (0, 1, 7, 1000):
        assert L.grt_photon_block_bytes(n) == 146 * n
        pa = abi.PhotonArrays.block(n)
        soa = abi.PhotonSoA()
        assert L.grt_host_photon_layout(C.c_void_p(pa._buffer.ctypes.data), n, C.byref(soa)) == 0
        mine = pa.soa()
        for f in abi.PHOTON_FIELDS:
            a = C.cast(getattr(soa, f), C.c_void_p).value
            b = C.cast(getattr(mine, f), C.c_void_p).value
            assert a == b, (n, f)
        if n:
            pa.x0[:] = np.arange(n)
            assert np.array_equal(pa.x0, np.arange(n)) and not pa.x1.any()
