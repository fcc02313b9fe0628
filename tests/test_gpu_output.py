"""Output-step archives (write_output_step, src/output/write_output.hpp:90-103)
through grt_run_with_output, the reference's whole step loop with its output.

Fixed-step RK4 and adaptive RK45 trajectories are bit-identical to the
reference's (the RK45 controller's pow rounds as glibc's does), so every
output-step archive must equal, byte for byte, the archive the reference's own
integrate_geodesics writes (oracle/_ref) for the same config -- the same files
(same output steps, same stop), members, dtypes, strides and values; the
image-products archive agrees to round-off (device atomics add in another
order).  An RK45 archive also equals the state after that many steps of a
separate run."""

import io
import zipfile

import numpy as np
import pytest

from grt import abi, config, torus, workloads
from helpers import mini

pytestmark = pytest.mark.gpu


def toml_with_output(p, tmp_path, variables, stride):
    torus_dir = tmp_path / "np"
    text = config.toml_text(p, str(torus_dir), str(tmp_path / "ref_out"), "grt")
    lines = [l for l in text.splitlines() if not l.startswith(("stride", "variables"))]
    at = lines.index("[output]") + 1
    lines[at:at] = [f"stride = {stride}", f'variables = "{variables}"']
    path = tmp_path / "c.toml"
    path.write_text("\n".join(lines) + "\n")
    return path


def reference_archives(reference, p, w, tmp_path, variables, stride):
    torus.write_numpy_dir(w.torus(), tmp_path / "np")
    toml = toml_with_output(p, tmp_path, variables, stride)
    ph = reference.init_image_photons(toml, w.pixels, w.pixels)
    reference.run(toml, ph, p, output_dir=tmp_path / "ref_out")
    return tmp_path / "ref_out"


def our_archives(gpu, p, w, out_dir, variables, stride, split=True):
    ctx = gpu.Context(p)
    try:
        ctx.set_launch_config(split_legs=int(split))
        ctx.upload_grid(w.torus())
        ctx.init_image_photons(w.pixels, w.pixels)
        st = ctx.run_with_output(out_dir, "grt", variables, stride)
        final = ctx.download_photons()
    finally:
        ctx.close()
    return st, final


def members(path):
    with zipfile.ZipFile(path) as z:
        return [(i.filename, z.read(i.filename)) for i in z.infolist()]


def step_of(name):
    return int(name.split("_step_")[1].split("_")[0])


def step_files(d):
    """Output-step archive names of directory d in step order."""
    return sorted((f.name for f in d.iterdir() if "_step_" in f.name), key=step_of)


ARCHIVE_CASES = [
    ("rk4", "all", 3), ("rk4", "id,frequency,x0,x1,x2,x3,k0,k1,k2,k3,I,Q,U,V,phase", 1),
    ("rk45", "all", 2), ("rk45", "x0,x1,x2,x3,k0,k1,k2,k3,dlambda,I,phase,terminate", 1),
]


@pytest.mark.parametrize("form,variables,stride", ARCHIVE_CASES)
def test_archives_are_the_references_bytes(gpu, reference, tmp_path, form, variables, stride):
    if form == "rk4":
        w = mini(workloads.C1, 16, (24, 16, 16), termination_percent=0.9, output_interval=37)
    else:
        w = mini(workloads.C2, 16, (32, 16, 16), termination_percent=0.9, output_interval=5)
    p = w.params()
    ref_dir = reference_archives(reference, p, w, tmp_path, variables, stride)
    ours = tmp_path / "ours"
    st, _ = our_archives(gpu, p, w, ours, variables, stride)
    files = step_files(ref_dir)
    assert len(files) > 2 and files == step_files(ours)
    for f in files:
        assert (ours / f).read_bytes() == (ref_dir / f).read_bytes(), f
    a = np.load(ours / "grt_image_products.npz")
    b = np.load(ref_dir / "grt_image_products.npz")
    assert list(a.keys()) == list(b.keys())
    for k in b.keys():
        assert a[k].dtype == b[k].dtype and a[k].shape == b[k].shape, k
        assert np.allclose(a[k], b[k], rtol=1e-12, atol=0.0), k
    last = step_of(files[-1])
    assert st["steps_done"] == last + 1


def test_rk45_archives(gpu, reference, tmp_path):
    w = mini(workloads.C2, 16, (32, 16, 16), output_interval=5)
    p = w.params()
    variables, stride = "all", 2
    ref_dir = reference_archives(reference, p, w, tmp_path, variables, stride)
    ours = tmp_path / "ours"
    st, final = our_archives(gpu, p, w, ours, variables, stride)
    files = step_files(ours)
    steps = [step_of(f) for f in files]
    assert steps == list(range(0, steps[-1] + 1, 5)) and st["steps_done"] == steps[-1] + 1
    # the reference's layout: members, dtypes, shapes (npy headers byte for byte)
    ref_layout = members(ref_dir / step_files(ref_dir)[0])
    our_layout = members(ours / files[0])
    assert [m[0] for m in our_layout] == [m[0] for m in ref_layout]
    for (_, ob), (_, rb) in zip(our_layout, ref_layout):
        hl = 10 + int.from_bytes(rb[8:10], "little")
        assert ob[:hl] == rb[:hl]
    # the last archive is the final state, strided
    z = np.load(ours / files[-1])
    for f in abi.PHOTON_FIELDS:
        assert np.array_equal(z[f], getattr(final, f)[::stride]), f
    # an intermediate archive is the state after that many steps
    mid = steps[len(steps) // 2]
    q = p.copy()
    q.max_steps = mid + 1
    ctx = gpu.Context(q)
    try:
        ctx.upload_grid(w.torus())
        ctx.init_image_photons(w.pixels, w.pixels)
        ctx.run()
        state = ctx.download_photons()
    finally:
        ctx.close()
    z = np.load(ours / f"grt_step_{mid}_rank0.npz")
    for f in abi.PHOTON_FIELDS:
        assert np.array_equal(z[f], getattr(state, f)[::stride]), f


def test_split_and_one_launch_write_the_same_archives(gpu, tmp_path):
    w = mini(workloads.C2, 12, (32, 16, 16), output_interval=3)
    p = w.params()
    our_archives(gpu, p, w, tmp_path / "a", "all", 1, split=True)
    our_archives(gpu, p, w, tmp_path / "b", "all", 1, split=False)
    files = step_files(tmp_path / "a")
    assert files == step_files(tmp_path / "b")
    for f in files:
        assert (tmp_path / "a" / f).read_bytes() == (tmp_path / "b" / f).read_bytes(), f


def test_write_output_step_directly(gpu, tmp_path):
    w = mini(workloads.C1, 8, (24, 16, 16))
    p = w.params()
    ctx = gpu.Context(p)
    try:
        ctx.upload_grid(w.torus())
        ctx.init_image_photons(8, 8)
        ctx.write_output_step_npz(tmp_path, "snap", 0, rank=3, variables="[phase, id, terminate]", stride=100)
        init = ctx.download_photons()
        with pytest.raises(Exception, match="unknown output variable: nope"):
            ctx.write_output_step_npz(tmp_path, "snap", 1, variables="id,nope")
        with pytest.raises(Exception, match="output.stride must be positive"):
            ctx.write_output_step_npz(tmp_path, "snap", 1, stride=0)
    finally:
        ctx.close()
    z = np.load(tmp_path / "snap_step_0_rank3.npz")
    assert list(z.keys()) == ["phase", "id", "terminate"]
    assert z["phase"].dtype == np.uint8 and z["id"].dtype == np.uint64 and z["terminate"].dtype == np.uint8
    assert np.array_equal(z["id"], init.id[:1]) and z["id"].shape == (1,)
    assert not (tmp_path / "snap_step_1_rank0.npz").exists()
