"""ctypes binding of lib/libgrt_b200.so (the C ABI declared in include/grt.h).

The product path is: Python (or any C caller) -> C ABI -> sm_100a kernels.
Nothing here computes physics; if the shared library is missing the import
fails loudly instead of falling back to anything else.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

from .abi import (GRT_OK, STATUS_NAMES, DeviceGrid, ImageProducts, ImageSpec, LaunchConfig, Params,
                  PhotonArrays, PhotonSoA, ProductArrays, RunStats)

PKG_ROOT = Path(__file__).resolve().parent.parent
LIB_PATH = PKG_ROOT / "lib" / "libgrt_b200.so"


class GrtError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


def build(jobs: int = 4) -> Path:
    """Compile the CUDA library for sm_100a (nvcc; no GPU needed)."""
    subprocess.run(["make", "-s", "-j", str(jobs), "-C", str(PKG_ROOT)], check=True)
    return LIB_PATH


_lib = None


def load(path: Path | None = None):
    """Load the shared library once and declare every entry point of grt.h."""
    global _lib
    if _lib is not None:
        return _lib
    path = Path(path or os.environ.get("GRT_LIB", LIB_PATH))
    if not path.exists():
        raise FileNotFoundError(f"{path} is not built; run grt.lib.build() (nvcc, sm_100a)")
    L = C.CDLL(str(path))
    vp = C.c_void_p
    P = C.POINTER
    L.grt_abi_version.restype = C.c_int32
    L.grt_build_info.restype = C.c_char_p
    L.grt_params_default.argtypes = [P(Params)]
    L.grt_params_default.restype = None
    L.grt_params_validate.argtypes = [P(Params), C.c_char_p, C.c_size_t]
    L.grt_create.argtypes = [P(Params), P(vp)]
    L.grt_destroy.argtypes = [vp]
    L.grt_destroy.restype = None
    L.grt_last_error.argtypes = [vp]
    L.grt_last_error.restype = C.c_char_p
    L.grt_set_params.argtypes = [vp, P(Params)]
    L.grt_set_stream.argtypes = [vp, vp]
    L.grt_synchronize.argtypes = [vp]
    L.grt_upload_grid.argtypes = [vp, C.c_size_t, C.c_size_t, C.c_size_t] + [P(C.c_double)] * 7
    L.grt_upload_grid_numpy_dir.argtypes = [vp, C.c_char_p]
    L.grt_upload_photons.argtypes = [vp, P(PhotonSoA), C.c_size_t]
    L.grt_init_image_photons.argtypes = [vp, C.c_uint64, C.c_uint64, C.c_uint64]
    L.grt_init_image_photons_random.argtypes = [vp, C.c_uint64, C.c_uint64]
    L.grt_run.argtypes = [vp, P(RunStats)]
    L.grt_download_photons.argtypes = [vp, P(PhotonSoA)]
    L.grt_photon_count.argtypes = [vp]
    L.grt_photon_count.restype = C.c_size_t
    L.grt_geodesic_count.argtypes = [vp]
    L.grt_geodesic_count.restype = C.c_uint64
    L.grt_products_block_bytes.argtypes = [vp]
    L.grt_products_block_bytes.restype = C.c_size_t
    L.grt_copy_products_block.argtypes = [vp, vp, C.c_size_t]
    L.grt_copy_products_block.restype = C.c_int
    L.grt_get_image_products.argtypes = [vp, P(ImageProducts)]
    L.grt_write_image_products_npz.argtypes = [vp, C.c_char_p, C.c_char_p]
    L.grt_get_launch_config.argtypes = [vp, P(LaunchConfig)]
    L.grt_set_launch_config.argtypes = [vp, P(LaunchConfig)]
    L.grt_measure_fma_peaks.argtypes = [P(C.c_double), P(C.c_double)]
    L.grt_trace_device_noalloc.argtypes = [P(Params), P(DeviceGrid), P(PhotonSoA), C.c_uint64, P(RunStats),
                                           vp, C.c_char_p, C.c_size_t]
    L.grt_init_image_batch.argtypes = [vp, P(ImageSpec), C.c_size_t, C.c_uint64]
    L.grt_batch_image_count.argtypes = [vp]
    L.grt_batch_image_count.restype = C.c_size_t
    L.grt_get_batch_image_products.argtypes = [vp, C.c_size_t, P(ImageProducts)]
    L.grt_write_batch_products_npz.argtypes = [vp, C.c_char_p, C.c_char_p]
    L.grt_render_graph.argtypes = [vp, P(RunStats)]
    L.grt_set_channel_sharing.argtypes = [vp, C.c_int]
    L.grt_set_channel_sharing.restype = C.c_int
    L.grt_init_image_rows.argtypes = [vp, C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64]
    L.grt_init_image_rows.restype = C.c_int
    L.grt_init_disk_photons.argtypes = [vp, C.c_uint64, P(C.c_uint64)]
    L.grt_init_disk_photons.restype = C.c_int
    L.grt_init_image_forward_photons.argtypes = [vp, C.c_uint64, C.c_uint64, C.c_double, C.c_uint64]
    L.grt_init_image_forward_photons.restype = C.c_int
    L.grt_set_cell_multipliers.argtypes = [vp, P(C.c_double), P(C.c_double)]
    L.grt_forward_checkpointed.argtypes = [vp, C.c_int64, P(RunStats)]
    L.grt_adjoint_image_I.argtypes = [vp, P(C.c_double), P(C.c_double), P(C.c_double)]
    L.grt_parse_output_variables.argtypes = [C.c_char_p, P(C.c_int32), P(C.c_size_t), C.c_char_p, C.c_size_t]
    L.grt_write_output_step_npz.argtypes = [vp, C.c_char_p, C.c_char_p, C.c_int64, C.c_int32, C.c_char_p, C.c_uint64]
    L.grt_run_with_output.argtypes = [vp, C.c_char_p, C.c_char_p, C.c_char_p, C.c_uint64, P(RunStats)]
    L.grt_get_all_batch_image_products.argtypes = [vp, P(ImageProducts), C.c_size_t]
    L.grt_get_all_batch_image_products.restype = C.c_int
    L.grt_photon_block_bytes.argtypes = [C.c_size_t]
    L.grt_photon_block_bytes.restype = C.c_size_t
    L.grt_host_photon_layout.argtypes = [vp, C.c_size_t, P(PhotonSoA)]
    L.grt_host_photon_layout.restype = C.c_int
    L.grt_render_async.argtypes = [vp, P(PhotonSoA), P(ImageProducts), C.c_size_t]
    L.grt_render_async.restype = C.c_int
    L.grt_render_wait.argtypes = [vp, P(RunStats)]
    L.grt_render_wait.restype = C.c_int
    for name in ("grt_parse_output_variables", "grt_write_output_step_npz",
                 "grt_run_with_output", "grt_set_cell_multipliers", "grt_forward_checkpointed", "grt_adjoint_image_I",
                 "grt_init_image_batch", "grt_get_batch_image_products", "grt_write_batch_products_npz",
                 "grt_render_graph", "grt_trace_device_noalloc", "grt_measure_fma_peaks", "grt_params_validate", "grt_create", "grt_set_params",
                 "grt_set_stream", "grt_synchronize", "grt_upload_grid", "grt_upload_grid_numpy_dir",
                 "grt_upload_photons", "grt_init_image_photons", "grt_init_image_photons_random", "grt_run",
                 "grt_download_photons",
                 "grt_get_image_products", "grt_write_image_products_npz", "grt_get_launch_config",
                 "grt_set_launch_config"):
        getattr(L, name).restype = C.c_int
    _lib = L
    return L


def default_params() -> Params:
    p = Params()
    load().grt_params_default(C.byref(p))
    return p


# The photon fields an output step can write, in the reference's order.
OUTPUT_FIELDS = ("id", "frequency", "emission_frame_energy", "x0", "x1", "x2", "x3", "k0", "k1", "k2", "k3",
                 "I", "Q", "U", "V", "dlambda", "terminate", "phase", "theta_disp", "phi_disp")
DEFAULT_OUTPUT_VARIABLES = "id,frequency,x0,x1,x2,x3,k0,k1,k2,k3,I,Q,U,V,phase"


def parse_output_variables(spec: str) -> list:
    """OutputSelection::parse: the field names an output step writes, in order."""
    fields = (C.c_int32 * (2 * len(OUTPUT_FIELDS)))()
    count = C.c_size_t(0)
    err = C.create_string_buffer(512)
    rc = load().grt_parse_output_variables(spec.encode(), fields, C.byref(count), err, 512)
    if rc != GRT_OK:
        raise GrtError(rc, err.value.decode())
    return [OUTPUT_FIELDS[fields[k]] for k in range(count.value)]


def validate_params(p: Params):
    buf = C.create_string_buffer(512)
    rc = load().grt_params_validate(C.byref(p), buf, 512)
    if rc != GRT_OK:
        raise GrtError(rc, buf.value.decode())


def measure_fma_peaks():
    """(fp64, fp32) FMA throughput of the current device in TFLOP/s."""
    d, f = C.c_double(), C.c_double()
    rc = load().grt_measure_fma_peaks(C.byref(d), C.byref(f))
    if rc != GRT_OK:
        raise GrtError(rc, "grt_measure_fma_peaks failed")
    return d.value, f.value


def trace_device_noalloc(params: Params, grid: DeviceGrid, photons: PhotonSoA, n: int, stream_ptr=None):
    """Allocation-free trace of n photons held in caller-owned device memory
    (photons: PhotonSoA of device pointers; grid: DeviceGrid of device
    pointers).  Returns the run statistics."""
    st = RunStats()
    err = C.create_string_buffer(512)
    rc = load().grt_trace_device_noalloc(C.byref(params), C.byref(grid) if grid is not None else None,
                                          C.byref(photons), n, C.byref(st), C.c_void_p(stream_ptr or 0), err, 512)
    if rc != GRT_OK:
        raise GrtError(rc, err.value.decode())
    return st.as_dict()


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Context:
    """One device context of the hot path (owns every device buffer)."""

    def __init__(self, params: Params):
        self.lib = load()
        self._h = C.c_void_p()
        self.params = params.copy()
        self._specs = []
        rc = self.lib.grt_create(C.byref(self.params), C.byref(self._h))
        if rc != GRT_OK:
            raise GrtError(rc, "grt_create failed (needs an sm_100 device and valid params)")

    def close(self):
        if self._h:
            self.lib.grt_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc):
        if rc != GRT_OK:
            raise GrtError(rc, self.lib.grt_last_error(self._h).decode())

    @property
    def handle(self):
        return self._h

    def set_params(self, p: Params):
        self.params = p.copy()
        self._check(self.lib.grt_set_params(self._h, C.byref(self.params)))

    def set_stream(self, stream_ptr: int | None):
        self._check(self.lib.grt_set_stream(self._h, C.c_void_p(stream_ptr or 0)))

    def synchronize(self):
        self._check(self.lib.grt_synchronize(self._h))

    def upload_grid(self, grid: dict | None):
        """grid: dict of the seven .npy arrays (name -> ndarray), or None for no fluid."""
        if grid is None:
            self._check(self.lib.grt_upload_grid(self._h, 0, 0, 0, *([None] * 7)))
            return
        keys = ("r.npy", "theta.npy", "phi.npy", "rho.npy", "Tgas.npy", "vel.npy", "mag.npy")
        arrs = [np.ascontiguousarray(grid[k], dtype=np.float64) for k in keys]
        nr, nth, nph = arrs[0].shape
        self._check(self.lib.grt_upload_grid(self._h, nr, nth, nph, *[_dp(a) for a in arrs]))

    def upload_grid_numpy_dir(self, path):
        self._check(self.lib.grt_upload_grid_numpy_dir(self._h, str(path).encode()))

    def upload_photons(self, ph: PhotonArrays):
        soa = ph.soa()
        self._check(self.lib.grt_upload_photons(self._h, C.byref(soa), ph.n))

    def init_image_photons(self, nx, ny, id_offset=0):
        self._check(self.lib.grt_init_image_photons(self._h, nx, ny, id_offset))

    def init_image_photons_random(self, n, id_offset=0):
        """n rays at the reference's random screen positions (Philox streams)."""
        self._check(self.lib.grt_init_image_photons_random(self._h, n, id_offset))

    def init_image_rows(self, nx, ny, row0, nrows, id_offset=0):
        """Pixel rows [row0, row0 + nrows) of the nx x ny screen (one image split across ranks)."""
        self._check(self.lib.grt_init_image_rows(self._h, nx, ny, row0, nrows, id_offset))

    def init_disk_photons(self, id_offset=0) -> int:
        """Disk-mode packets from every grid cell (initialize_photons_disk); returns their count."""
        n = C.c_uint64(0)
        self._check(self.lib.grt_init_disk_photons(self._h, id_offset, C.byref(n)))
        return int(n.value)

    def init_image_forward_photons(self, nx, ny, back_distance, id_offset=0):
        """Line-of-sight forward rays behind the scene, aimed at the camera."""
        self._check(self.lib.grt_init_image_forward_photons(self._h, nx, ny, float(back_distance), id_offset))

    def init_image_batch(self, specs, id_offset=0):
        """Rays of several images (list of ImageSpec) for one batched launch."""
        arr = (ImageSpec * len(specs))(*specs)
        self._check(self.lib.grt_init_image_batch(self._h, arr, len(specs), id_offset))
        self._specs = list(specs)

    def set_channel_sharing(self, enable: bool):
        """Frequency channels of a batch share their geodesics (default on)."""
        self._check(self.lib.grt_set_channel_sharing(self._h, int(bool(enable))))

    @property
    def batch_image_count(self) -> int:
        return int(self.lib.grt_batch_image_count(self._h))

    def batch_image_products(self, image: int, out: ProductArrays | None = None) -> ProductArrays:
        if out is None:
            # an index the library will reject still gets valid buffers to pass
            nx, ny = (self._specs[image].nx, self._specs[image].ny) if 0 <= image < len(self._specs) else (1, 1)
            out = ProductArrays(nx, ny, self.params.spectrum_bins)
        s = out.struct()
        self._check(self.lib.grt_get_batch_image_products(self._h, image, C.byref(s)))
        return out

    def all_batch_image_products(self, outs: list) -> list:
        """Every image's products (outs[k]: ProductArrays for image k) with one synchronisation."""
        arr = (ImageProducts * len(outs))(*[o.struct() for o in outs])
        self._check(self.lib.grt_get_all_batch_image_products(self._h, arr, len(outs)))
        return outs

    def write_batch_products_npz(self, output_dir, name):
        self._check(self.lib.grt_write_batch_products_npz(self._h, str(output_dir).encode(), name.encode()))

    def render_graph(self) -> dict:
        """Re-initialise, trace and build products through the context's CUDA graph."""
        st = RunStats()
        rc = self.lib.grt_render_graph(self._h, C.byref(st))
        self._check(rc)
        return st.as_dict()

    def render_async(self, photons: PhotonArrays, outs: list):
        """Enqueue a render of host photons (a PhotonArrays.block of the batch's
        count, pinned for overlap) into outs (ProductArrays per image); returns
        at once.  photons and outs stay in use until render_wait."""
        soa = photons.soa()
        arr = (ImageProducts * len(outs))(*[o.struct() for o in outs])
        self._check(self.lib.grt_render_async(self._h, C.byref(soa), arr, len(outs)))
        self._pending = (photons, outs, soa, arr)

    def render_wait(self) -> dict:
        """Wait for the render in flight; its products are then in its outs."""
        st = RunStats()
        rc = self.lib.grt_render_wait(self._h, C.byref(st))
        self._pending = None
        self._check(rc)
        return st.as_dict()

    # ---- differentiable radiative transfer ----
    def set_cell_multipliers(self, m_abs=None, m_emis=None):
        """Per-cell multipliers on dtau and dI (arrays of the grid's shape; None = 1)."""
        self._mult = [None if m is None else np.ascontiguousarray(m, dtype=np.float64).ravel()
                      for m in (m_abs, m_emis)]
        self._check(self.lib.grt_set_cell_multipliers(self._h, *[_dp(m) if m is not None else None
                                                                  for m in self._mult]))

    def forward_checkpointed(self, checkpoint_interval: int = 64) -> dict:
        st = RunStats()
        self._check(self.lib.grt_forward_checkpointed(self._h, int(checkpoint_interval), C.byref(st)))
        return st.as_dict()

    def adjoint_image_I(self, dL_dimage_I, grid_shape):
        """(dL/dm_abs, dL/dm_emis) of the last forward_checkpointed, each of grid_shape."""
        g = np.ascontiguousarray(dL_dimage_I, dtype=np.float64)
        if g.shape != (self.params.image_ny, self.params.image_nx):
            raise ValueError(f"dL/dimage_I must have shape {(self.params.image_ny, self.params.image_nx)}")
        ga = np.zeros(int(np.prod(grid_shape)))
        ge = np.zeros(int(np.prod(grid_shape)))
        self._check(self.lib.grt_adjoint_image_I(self._h, _dp(g), _dp(ga), _dp(ge)))
        return ga.reshape(grid_shape), ge.reshape(grid_shape)

    def run(self) -> dict:
        st = RunStats()
        rc = self.lib.grt_run(self._h, C.byref(st))
        self._check(rc)
        return st.as_dict()

    @property
    def n(self):
        return int(self.lib.grt_photon_count(self._h))

    @property
    def products_block_bytes(self):
        return int(self.lib.grt_products_block_bytes(self._h))

    def copy_products_block(self, dst_ptr: int, nbytes: int):
        """Enqueue a copy of every image's products into dst_ptr (device or host
        memory; see grt_copy_products_block) on the context's stream."""
        self._check(self.lib.grt_copy_products_block(self._h, C.c_void_p(dst_ptr), nbytes))

    @property
    def geodesics(self):
        """Geodesics a run traces (fewer than n when frequency channels share them)."""
        return int(self.lib.grt_geodesic_count(self._h))

    def download_photons(self, out: PhotonArrays | None = None) -> PhotonArrays:
        out = out or PhotonArrays(self.n)
        soa = out.soa()
        self._check(self.lib.grt_download_photons(self._h, C.byref(soa)))
        return out

    def image_products(self, out: ProductArrays | None = None) -> ProductArrays:
        out = out or ProductArrays.for_params(self.params)
        s = out.struct()
        self._check(self.lib.grt_get_image_products(self._h, C.byref(s)))
        return out

    def write_image_products_npz(self, output_dir, name):
        self._check(self.lib.grt_write_image_products_npz(self._h, str(output_dir).encode(), name.encode()))

    def write_output_step_npz(self, output_dir, name, step: int, rank: int = 0,
                              variables: str = DEFAULT_OUTPUT_VARIABLES, stride: int = 1):
        """<output_dir>/<name>_step_<step>_rank<rank>.npz of the current photons."""
        self._check(self.lib.grt_write_output_step_npz(self._h, str(output_dir).encode(), name.encode(), int(step),
                                                       int(rank), variables.encode(), int(stride)))

    def run_with_output(self, output_dir, name, variables: str = DEFAULT_OUTPUT_VARIABLES, stride: int = 1) -> dict:
        """The reference's step loop with an archive after every output step
        (and the image products at the end in image mode)."""
        st = RunStats()
        self._check(self.lib.grt_run_with_output(self._h, str(output_dir).encode(), name.encode(), variables.encode(),
                                                 int(stride), C.byref(st)))
        return st.as_dict()

    def launch_config(self) -> dict:
        lc = LaunchConfig()
        self._check(self.lib.grt_get_launch_config(self._h, C.byref(lc)))
        return lc.as_dict()

    def set_launch_config(self, **kw):
        lc = LaunchConfig()
        self._check(self.lib.grt_get_launch_config(self._h, C.byref(lc)))
        for k, v in kw.items():
            setattr(lc, k, int(v))
        self._check(self.lib.grt_set_launch_config(self._h, C.byref(lc)))
