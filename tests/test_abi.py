"""The C ABI boundary without a GPU: the library loads, exports every
function include/grt.h declares, its structs have the ctypes layout, and the
TOML mirror parses configs exactly like the reference's own loader."""

import ctypes as C
import re
import subprocess

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
def test_adapter_maps_the_reference_loader(reference, tmp_path, case):
    """include/grt_reference_adapter.hpp maps the structs the reference's own
    TOML loader fills (and the reference's runtime globals) onto grt_params:
    equal, field by field, to the params the config was written from, and to
    the test-side mapping in oracle/ref_driver.cpp."""
    p = _toml_cases()[case]
    t = config.write_toml(p, tmp_path / "c.toml", tmp_path / "np", tmp_path / "out", name="run")
    mine = reference.adapter_params_from_toml(t)
    ref = reference.params_from_toml(t)
    for k, v in ref.as_dict().items():
        assert getattr(mine, k) == v, k
    for k, v in p.as_dict().items():
        if k in ("precision", "rank"):
            continue
        assert getattr(mine, k) == v, k
    lib.validate_params(mine)


def test_adapter_on_reference_example_configs(reference):
    root = pyoracle.Reference.root()
    cfgs = sorted((root / "config").glob("*.toml")) if root else []
    if not cfgs:
        pytest.skip("the reference tree oracle/_ref was built from is not on this machine")
    for t in cfgs:
        mine = reference.adapter_params_from_toml(t)
        ref = reference.params_from_toml(t)
        for k, v in ref.as_dict().items():
            assert getattr(mine, k) == v, (t.name, k)
        lib.validate_params(mine)


@pytest.mark.parametrize("field,value,msg", [
    ("spin", 2.0, "grt_params.spin: |spin| <= mass"),
    ("integrator", 7, "grt_params.integrator"),
    ("termination_percent", 1.5, "termination_percent: in (0, 1]"),
    ("generator", 9, "grt_params.generator"),
    ("output_interval", 0, "output_interval: positive"),
    ("r_term_max", 0.5, "termination radii"),
    ("rtol", float("nan"), "atol, rtol"),
    ("spectrum_min_hz", 1e30, "spectrum range"),
])
def test_param_validation_names_the_field(field, value, msg):
    p = workloads.C2.params()
    setattr(p, field, value)
    with pytest.raises(lib.GrtError, match=re.escape(msg)):
        lib.validate_params(p)


def test_param_validation():
    p = workloads.C2.params()
    lib.validate_params(p)
    p.camera_distance = -1.0
    with pytest.raises(lib.GrtError, match="camera: distance"):
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
