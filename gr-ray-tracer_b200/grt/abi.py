"""ctypes mirror of include/grt.h (the C ABI of the hot path).

Structures here must match grt.h field for field; tests/test_abi.py checks the
sizes against the compiled library.  Numpy-backed helpers allocate the host
arrays a call needs and build the pointer structs from them.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

GRT_OK, GRT_EINVAL, GRT_ECUDA, GRT_ENOMEM, GRT_ESTATE, GRT_ETIMEOUT, GRT_EIO, GRT_ENODEV = range(8)
STATUS_NAMES = {0: "GRT_OK", 1: "GRT_EINVAL", 2: "GRT_ECUDA", 3: "GRT_ENOMEM", 4: "GRT_ESTATE",
                5: "GRT_ETIMEOUT", 6: "GRT_EIO", 7: "GRT_ENODEV"}

MODE_IMAGE, MODE_DISK = 0, 1
RK4, RK45 = 0, 1
GEN_BLACKBODY, GEN_POWER_LAW, GEN_CUSTOM = 0, 1, 2
PHASE_DISK, PHASE_BACKWARD, PHASE_FORWARD, PHASE_ARRIVED, PHASE_REJECTED = 0, 1, 2, 3, 4
PREC_FP64, PREC_MIXED, PREC_MIXED_GRID = 0, 1, 2

_D, _I32, _I64, _U64 = C.c_double, C.c_int32, C.c_int64, C.c_uint64


class Params(C.Structure):
    _fields_ = [
        ("mode", _I32), ("integrator", _I32), ("precision", _I32), ("generator", _I32),
        ("mass", _D), ("spin", _D), ("r_term_min", _D), ("r_term_max", _D),
        ("atol", _D), ("rtol", _D), ("min_step_scale", _D), ("max_step_scale", _D), ("safety", _D),
        ("max_steps", _I64), ("termination_percent", _D), ("output_interval", _U64),
        ("nphotons", _U64), ("initial_step", _D),
        ("camera_distance", _D), ("camera_theta", _D), ("camera_phi", _D),
        ("camera_width", _D), ("camera_height", _D),
        ("absorption_enabled", _I32), ("emission_enabled", _I32),
        ("absorption_coefficient", _D), ("emission_coefficient", _D),
        ("scattering_enabled", _I32), ("rank", _I32),
        ("scattering_albedo", _D), ("scattering_seed", _U64),
        ("superphoton_count_normalization", _D), ("energy_per_cell_erg", _D),
        ("power_law_slope", _D), ("nu_min_hz", _D), ("nu_max_hz", _D), ("custom_frequency_hz", _D),
        ("length_cm_per_code", _D), ("time_s_per_code", _D), ("density_g_cm3_per_code", _D),
        ("temperature_k_per_code", _D), ("four_velocity_cm_s_per_code", _D),
        ("magnetic_gauss_per_code", _D),
        ("image_nx", _U64), ("image_ny", _U64), ("spectrum_bins", _U64),
        ("spectrum_min_hz", _D), ("spectrum_max_hz", _D),
    ]

    def copy(self) -> "Params":
        other = Params()
        C.pointer(other)[0] = self
        return other

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}

    def update(self, **kw):
        for k, v in kw.items():
            if not hasattr(self, k):
                raise AttributeError(f"grt_params has no field {k!r}")
            setattr(self, k, v)
        return self


_DP = C.POINTER(C.c_double)
_U8P = C.POINTER(C.c_uint8)
_U64P = C.POINTER(C.c_uint64)

PHOTON_FIELDS = ("id", "frequency", "emission_frame_energy", "x0", "x1", "x2", "x3",
                 "k0", "k1", "k2", "k3", "I", "Q", "U", "V", "dlambda", "theta_disp",
                 "phi_disp", "terminate", "phase")
PHOTON_DTYPES = {"id": np.uint64, "terminate": np.uint8, "phase": np.uint8}


class PhotonSoA(C.Structure):
    _fields_ = [("id", _U64P)] + [(n, _DP) for n in PHOTON_FIELDS[1:18]] + [
        ("terminate", _U8P), ("phase", _U8P)]


class DeviceGrid(C.Structure):
    """grt_device_grid: the seven grid arrays as device pointers (reference layout)."""
    _fields_ = [("nr", _U64), ("ntheta", _U64), ("nphi", _U64)] + [
        (n, C.c_void_p) for n in ("r", "theta", "phi", "rho", "temperature", "vel4", "mag4")]


class RunStats(C.Structure):
    _fields_ = [("steps_done", _I64), ("n_terminated", _U64), ("accepted_steps", _U64),
                ("rejected_attempts", _U64), ("photon_calls", _U64), ("launches", _U64),
                ("trace_ms", _D), ("timed_out", _I32), ("pad", _I32)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_ if name != "pad"}


class ImageProducts(C.Structure):
    _fields_ = [("image_I", _DP), ("image_Q", _DP), ("image_U", _DP), ("image_V", _DP),
                ("spectrum_frequency_hz", _DP), ("spectrum_I", _DP), ("arrived_count", _U64P)]


class LaunchConfig(C.Structure):
    _fields_ = [("threads_per_block", _I32), ("blocks_per_sm", _I32),
                ("refill_threshold", _I32), ("photons_per_grab", _I32), ("split_legs", _I32),
                ("pad", _I32), ("max_iterations", C.c_int64)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class ImageSpec(C.Structure):
    """grt_image_spec: one image of a batched launch."""
    _fields_ = [("camera_theta", _D), ("camera_phi", _D), ("camera_distance", _D), ("camera_width", _D),
                ("camera_height", _D), ("nx", _U64), ("ny", _U64), ("custom_frequency_hz", _D),
                ("absorption_coefficient", _D), ("emission_coefficient", _D)]

    @classmethod
    def from_params(cls, p: Params, nx: int, ny: int, **kw) -> "ImageSpec":
        sp = cls(camera_theta=p.camera_theta, camera_phi=p.camera_phi, camera_distance=p.camera_distance,
                 camera_width=p.camera_width, camera_height=p.camera_height, nx=nx, ny=ny,
                 custom_frequency_hz=p.custom_frequency_hz, absorption_coefficient=p.absorption_coefficient,
                 emission_coefficient=p.emission_coefficient)
        for k, v in kw.items():
            if not hasattr(sp, k):
                raise AttributeError(f"grt_image_spec has no field {k!r}")
            setattr(sp, k, v)
        return sp

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


def _ptr(arr, ctype):
    return arr.ctypes.data_as(C.POINTER(ctype))


class PhotonArrays:
    """Numpy-owned host SoA of n photons (one array per Photons field)."""

    def __init__(self, n: int):
        self.n = int(n)
        for f in PHOTON_FIELDS:
            setattr(self, f, np.zeros(self.n, dtype=PHOTON_DTYPES.get(f, np.float64)))

    @classmethod
    def block(cls, n: int, buffer=None):
        """The SoA as views into one byte buffer of 146 n bytes in the layout of
        grt_host_photon_layout (id, the 17 doubles, terminate, phase back to
        back), which grt_upload_photons / grt_download_photons move with one
        transfer.  `buffer` (e.g. a pinned tensor's numpy view) or a new array."""
        n = int(n)
        buf = np.zeros(146 * n, dtype=np.uint8) if buffer is None else buffer
        if buf.size < 146 * n or buf.ctypes.data % 8:
            raise ValueError("the buffer needs 146 * n bytes, 8-byte aligned")
        pa = cls.__new__(cls)
        pa.n = n
        pa._buffer = buf
        for k, f in enumerate(PHOTON_FIELDS):
            off = 8 * n * k if k <= 17 else 144 * n + n * (k - 18)
            size = 8 if k <= 17 else 1
            setattr(pa, f, buf[off:off + size * n].view(PHOTON_DTYPES.get(f, np.float64)))
        return pa

    @classmethod
    def from_dict(cls, d):
        n = len(d["x0"])
        pa = cls(n)
        for f in PHOTON_FIELDS:
            getattr(pa, f)[:] = d[f]
        return pa

    def as_dict(self):
        return {f: getattr(self, f) for f in PHOTON_FIELDS}

    def copy(self):
        return PhotonArrays.from_dict({f: getattr(self, f).copy() for f in PHOTON_FIELDS})

    def soa(self) -> PhotonSoA:
        s = PhotonSoA()
        s.id = _ptr(self.id, C.c_uint64)
        for f in PHOTON_FIELDS[1:18]:
            setattr(s, f, _ptr(getattr(self, f), C.c_double))
        s.terminate = _ptr(self.terminate, C.c_uint8)
        s.phase = _ptr(self.phase, C.c_uint8)
        return s


class ProductArrays:
    """Numpy-owned host buffers for one set of image products."""

    def __init__(self, nx: int, ny: int, bins: int):
        self.nx, self.ny, self.bins = int(nx), int(ny), int(bins)
        self.image_I = np.zeros((self.ny, self.nx))
        self.image_Q = np.zeros((self.ny, self.nx))
        self.image_U = np.zeros((self.ny, self.nx))
        self.image_V = np.zeros((self.ny, self.nx))
        self.spectrum_frequency_hz = np.zeros(self.bins)
        self.spectrum_I = np.zeros(self.bins)
        self.arrived_count = np.zeros(1, dtype=np.uint64)

    @classmethod
    def for_params(cls, p: Params):
        return cls(p.image_nx, p.image_ny, p.spectrum_bins)

    def struct(self) -> ImageProducts:
        s = ImageProducts()
        for f in ("image_I", "image_Q", "image_U", "image_V", "spectrum_frequency_hz", "spectrum_I"):
            setattr(s, f, _ptr(getattr(self, f), C.c_double))
        s.arrived_count = _ptr(self.arrived_count, C.c_uint64)
        return s

    def as_dict(self):
        return {f: getattr(self, f) for f in ("image_I", "image_Q", "image_U", "image_V",
                                               "spectrum_frequency_hz", "spectrum_I", "arrived_count")}
