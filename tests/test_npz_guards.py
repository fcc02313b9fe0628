"""The NPZ writer (grt::NpzOut, the format of the reference's cnpy NpzWriter:
a stored ZIP without the ZIP64 extension) refuses an archive whose member
size, member offset or central directory outgrows its 32-bit fields, as the
reference does (src/cnpy.h:176-181, 220-248), instead of wrapping them.  The
32-bit limit is lowered here so the test needs kilobytes, not 4 GiB; the
archive written below the limit is read back by numpy."""

import subprocess

import numpy as np
import pytest

from conftest import PKG

SRC = r"""
#include <cstdio>
#include "grt_host.h"
int main(int argc, char** argv) {
    const std::vector<size_t> shape{100};
    std::vector<double> v(100);
    for (int i = 0; i < 100; ++i) v[i] = i;
    const auto payload = grt::npy_bytes("<f8", shape, v.data(), 8);
    const uint64_t P = payload.size();
    const uint64_t M = 30 + 6 + P;  // a member "mK.npy" with its local header
    // 1. below the limit: a valid archive
    {
        grt::NpzOut z(4096);
        if (!z.open(argv[1]) || !z.add("a", payload) || !z.add("b", payload) || !z.close()) return 1;
    }
    // 2. a member larger than the limit
    {
        grt::NpzOut z(P - 1);
        z.open(argv[2]);
        if (z.add("a", payload)) return 2;
        std::printf("member: %s\n", z.error().c_str());
    }
    // 3. a member offset beyond the limit (the sixth member starts past it)
    {
        grt::NpzOut z(4 * M);
        z.open(argv[2]);
        int k = 0;
        while (k < 10 && z.add("m" + std::to_string(k), payload)) ++k;
        std::printf("offset: %d added; %s\n", k, z.error().c_str());
        if (k != 5) return 3;
    }
    // 4. the central directory beyond the limit
    {
        grt::NpzOut z(P + 1);  // the member fits; the directory starts at 35 + P
        z.open(argv[2]);
        if (!z.add("a", payload)) return 4;
        if (z.close()) return 5;
        std::printf("directory: %s\n", z.error().c_str());
    }
    return 0;
}
"""


def test_npz_writer_refuses_archives_beyond_32_bit_fields(tmp_path):
    src = tmp_path / "t.cpp"
    src.write_text(SRC)
    exe = tmp_path / "t"
    csrc = PKG / "csrc"
    r = subprocess.run(["g++", "-std=c++17", "-O1", f"-I{csrc}", f"-I{PKG.parent / 'include'}", str(src),
                        str(csrc / "grt_host.cpp"), "-o", str(exe)], capture_output=True, text=True)
    if r.returncode != 0:
        pytest.fail(r.stderr[-2000:])
    good, bad = tmp_path / "good.npz", tmp_path / "bad.npz"
    out = subprocess.run([str(exe), str(good), str(bad)], capture_output=True, text=True)
    assert out.returncode == 0, (out.returncode, out.stdout)
    lines = out.stdout.splitlines()
    assert lines == ["member: NumPy archive exceeds the non-ZIP64 size limit",
                     "offset: 5 added; NumPy archive exceeds the non-ZIP64 size limit",
                     "directory: NumPy archive exceeds the non-ZIP64 size limit"]
    z = np.load(good)
    assert list(z.keys()) == ["a", "b"]
    assert np.array_equal(z["b"], np.arange(100.0))
