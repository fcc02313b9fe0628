"""ORACLE -- TEST INFRASTRUCTURE ONLY.

ctypes bindings for the two CPU checkers built by oracle/Makefile:
  * liboracle.so        -- the project's restatement of the reference hot path;
  * _ref/libgrt_ref.so  -- the reference's own code compiled against oracle/shim.
Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg import this.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
sys.path.insert(0, str(ROOT / "gr-ray-tracer_b200"))

from grt.abi import ImageProducts, Params, PhotonArrays, PhotonSoA, ProductArrays, RunStats  # noqa: E402

ORACLE_SO = HERE / "liboracle.so"
REF_SO = HERE / "_ref" / "libgrt_ref.so"

_DP = C.POINTER(C.c_double)


def build(with_ref=None):
    """Build the oracle (and the reference driver when the reference tree exists)."""
    target = ["all"] if with_ref is None else (["oracle", "ref"] if with_ref else ["oracle"])
    subprocess.run(["make", "-s", "-C", str(HERE)] + target, check=True)


def _dp(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(_DP)


class Oracle:
    def __init__(self, path=ORACLE_SO):
        if not Path(path).exists():
            build(with_ref=False)
        self.lib = C.CDLL(str(path))
        L = self.lib
        P = C.POINTER(Params)
        L.oracle_run.argtypes = [P, C.c_size_t, C.c_size_t, C.c_size_t] + [_DP] * 9 + [
            C.POINTER(PhotonSoA), C.c_size_t, C.POINTER(RunStats)]
        L.oracle_init_image_photons.argtypes = [P, C.c_uint64, C.c_uint64, C.c_uint64, C.POINTER(PhotonSoA)]
        L.oracle_init_image_photons_random.argtypes = [P, C.c_uint64, C.c_uint64, C.POINTER(PhotonSoA)]
        L.oracle_image_products.argtypes = [P, C.POINTER(PhotonSoA), C.c_size_t, C.POINTER(ImageProducts)]
        L.oracle_hamiltonian_rhs.argtypes = [_DP, _DP, C.c_double, C.c_double, _DP]
        L.oracle_compute_r.argtypes = [C.c_double] * 4
        L.oracle_compute_r.restype = C.c_double
        L.oracle_metric.argtypes = [_DP, C.c_double, C.c_double, _DP]
        L.oracle_inverse_metric.argtypes = [_DP, C.c_double, C.c_double, _DP]
        L.oracle_inverse_metric_deriv.argtypes = [_DP, C.c_double, C.c_double, _DP]
        L.oracle_null_momentum.argtypes = [_DP, _DP, C.c_double, C.c_double, _DP]
        L.oracle_norm.argtypes = [_DP, _DP, C.c_double, C.c_double]
        L.oracle_norm.restype = C.c_double
        L.oracle_rk4_step.argtypes = [P, _DP, C.c_double]
        L.oracle_rk45_step.argtypes = [P, _DP, _DP]
        L.oracle_locate_cell.argtypes = [C.c_size_t] * 3 + [_DP] * 3 + [C.c_double] * 3 + [C.POINTER(C.c_int)]
        L.oracle_sample_fluid.argtypes = [P] + [C.c_size_t] * 3 + [_DP] * 7 + [_DP, _DP, _DP, C.POINTER(C.c_int)]
        L.oracle_apply_rt.argtypes = [_DP] + [C.c_double] * 4 + [C.c_int, C.c_int, C.c_double, C.c_double]
        L.oracle_philox_block.argtypes = [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
        L.oracle_philox_drand.argtypes = [C.c_uint64, C.c_uint64, C.c_uint32, C.c_int]
        L.oracle_philox_drand.restype = C.c_double
        L.oracle_set_pow_mode.argtypes = [C.c_int]
        L.oracle_pow_quarter_pair.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p]
        L.oracle_pow_quarter_pair.restype = None
        L.oracle_observation_bin.argtypes = [C.c_double, C.c_double, C.c_double, C.c_uint64]
        L.oracle_observation_bin.restype = C.c_uint64
        L.oracle_init_disk_photons.argtypes = ([P] + [C.c_size_t] * 3 + [_DP] * 7 +
                                               [C.c_uint64, C.POINTER(PhotonSoA), C.POINTER(C.c_uint64)])
        L.oracle_det_sincos.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p]
        L.oracle_det_sincos.restype = None
        L.oracle_init_forward_photons.argtypes = [P, C.c_uint64, C.c_uint64, C.c_double, C.c_uint64,
                                                  C.POINTER(PhotonSoA)]
        L.oracle_adjoint_image_I.argtypes = ([P] + [C.c_size_t] * 3 + [_DP] * 9 +
                                             [C.POINTER(PhotonSoA), C.c_size_t, _DP, _DP, _DP])

    def set_pow_mode(self, mode):
        """The RK45 controller's pow(1/err, 0.25): 'libm' (default) calls
        std::pow like the reference's host build; 'restated' calls the
        kernels' grt::pow_quarter compiled for the host."""
        self.lib.oracle_set_pow_mode({"libm": 0, "restated": 1}[mode])

    # ---- whole-path entry points ----
    def init_image_photons(self, p: Params, nx, ny, id_offset=0) -> PhotonArrays:
        ph = PhotonArrays(nx * ny)
        soa = ph.soa()
        self.lib.oracle_init_image_photons(C.byref(p), nx, ny, id_offset, C.byref(soa))
        return ph

    def init_image_photons_random(self, p: Params, n, id_offset=0) -> PhotonArrays:
        ph = PhotonArrays(n)
        soa = ph.soa()
        self.lib.oracle_init_image_photons_random(C.byref(p), n, id_offset, C.byref(soa))
        return ph

    def init_disk_photons(self, p: Params, grid: dict, id_offset=0) -> PhotonArrays:
        r = grid["r.npy"]
        nr, nth, nph = r.shape
        keep = [np.ascontiguousarray(grid[k], dtype=np.float64) for k in
                ("r.npy", "theta.npy", "phi.npy", "rho.npy", "Tgas.npy", "vel.npy", "mag.npy")]
        n = C.c_uint64(0)
        self.lib.oracle_init_disk_photons(C.byref(p), nr, nth, nph, *[_dp(a) for a in keep], id_offset, None,
                                          C.byref(n))
        ph = PhotonArrays(n.value)
        soa = ph.soa()
        self.lib.oracle_init_disk_photons(C.byref(p), nr, nth, nph, *[_dp(a) for a in keep], id_offset,
                                          C.byref(soa), C.byref(n))
        return ph

    def init_forward_photons(self, p: Params, nx, ny, back, id_offset=0) -> PhotonArrays:
        ph = PhotonArrays(nx * ny)
        soa = ph.soa()
        self.lib.oracle_init_forward_photons(C.byref(p), nx, ny, C.c_double(back), id_offset, C.byref(soa))
        return ph

    def run(self, p: Params, grid: dict, photons: PhotonArrays, m_abs=None, m_emis=None):
        """Trace photons in place with the reference step loop; returns stats dict."""
        r = grid["r.npy"]
        nr, nth, nph = r.shape
        keep = [np.ascontiguousarray(grid[k], dtype=np.float64) for k in
                ("r.npy", "theta.npy", "phi.npy", "rho.npy", "Tgas.npy", "vel.npy", "mag.npy")]
        ma = None if m_abs is None else np.ascontiguousarray(m_abs, dtype=np.float64)
        me = None if m_emis is None else np.ascontiguousarray(m_emis, dtype=np.float64)
        st = RunStats()
        soa = photons.soa()
        self.lib.oracle_run(C.byref(p), nr, nth, nph, *[_dp(a) for a in keep], _dp(ma), _dp(me),
                            C.byref(soa), photons.n, C.byref(st))
        return st.as_dict()

    def adjoint_image_I(self, p: Params, grid: dict, photons: PhotonArrays, dL_dI, m_abs=None, m_emis=None):
        """FP64 reference gradient of a Stokes-I image loss: traces photons in
        place and returns (dL/dm_abs, dL/dm_emis) over the grid cells."""
        r = grid["r.npy"]
        nr, nth, nph = r.shape
        keep = [np.ascontiguousarray(grid[k], dtype=np.float64) for k in
                ("r.npy", "theta.npy", "phi.npy", "rho.npy", "Tgas.npy", "vel.npy", "mag.npy")]
        ma = None if m_abs is None else np.ascontiguousarray(m_abs, dtype=np.float64).ravel()
        me = None if m_emis is None else np.ascontiguousarray(m_emis, dtype=np.float64).ravel()
        g = np.ascontiguousarray(dL_dI, dtype=np.float64)
        if g.shape != (p.image_ny, p.image_nx):
            raise ValueError(f"dL_dI must have shape {(p.image_ny, p.image_nx)}")
        ga = np.zeros(nr * nth * nph)
        ge = np.zeros(nr * nth * nph)
        soa = photons.soa()
        self.lib.oracle_adjoint_image_I(C.byref(p), nr, nth, nph, *[_dp(a) for a in keep], _dp(ma), _dp(me),
                                        C.byref(soa), photons.n, _dp(g), _dp(ga), _dp(ge))
        return ga.reshape(r.shape), ge.reshape(r.shape)

    def image_products(self, p: Params, photons: PhotonArrays) -> ProductArrays:
        out = ProductArrays.for_params(p)
        s = out.struct()
        soa = photons.soa()
        self.lib.oracle_image_products(C.byref(p), C.byref(soa), photons.n, C.byref(s))
        return out

    # ---- unit-level ----
    def rhs(self, X, P, a, M):
        out = np.zeros(8)
        self.lib.oracle_hamiltonian_rhs(_dp(np.asarray(X, float)), _dp(np.asarray(P, float)), a, M, _dp(out))
        return out

    def null_momentum(self, X, K, a, M):
        out = np.zeros(4)
        ok = self.lib.oracle_null_momentum(_dp(np.asarray(X, float)), _dp(np.asarray(K, float)), a, M, _dp(out))
        return bool(ok), out

    def locate_cell(self, r, th, ph, radius, polar, azimuth):
        r = np.ascontiguousarray(r, float); th = np.ascontiguousarray(th, float); ph = np.ascontiguousarray(ph, float)
        ijk = (C.c_int * 3)()
        ok = self.lib.oracle_locate_cell(*r.shape, _dp(r), _dp(th), _dp(ph), radius, polar, azimuth, ijk)
        return bool(ok), tuple(ijk)


class Reference:
    """The reference's own code (shim-compiled).  Needs oracle/_ref/libgrt_ref.so."""

    def __init__(self, path=REF_SO):
        if not Path(path).exists():
            raise FileNotFoundError(f"{path} is not built (needs the reference tree at build time)")
        self.lib = C.CDLL(str(path))
        L = self.lib
        L.ref_last_error.restype = C.c_char_p
        L.ref_params_from_toml.argtypes = [C.c_char_p, C.POINTER(Params)]
        L.ref_adapter_params_from_toml.argtypes = [C.c_char_p, C.POINTER(Params)]
        L.ref_init_image_photons.argtypes = [C.c_char_p, C.c_uint64, C.c_uint64, C.c_uint64, C.POINTER(PhotonSoA)]
        L.ref_init_image_photons_random.argtypes = [C.c_char_p, C.c_uint64, C.c_uint64, C.POINTER(PhotonSoA)]
        L.ref_run_photons.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p, C.POINTER(PhotonSoA), C.c_uint64,
                                      C.POINTER(ImageProducts), _DP, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
        L.ref_init_disk_photons.argtypes = [C.c_char_p, C.c_char_p, C.c_uint64, C.POINTER(PhotonSoA),
                                            C.POINTER(C.c_uint64)]
        L.ref_hamiltonian_rhs.argtypes = [_DP, _DP, C.c_double, C.c_double, _DP]
        L.ref_null_momentum.argtypes = [_DP, _DP, C.c_double, C.c_double, _DP]
        L.ref_inverse_metric_deriv.argtypes = [_DP, C.c_double, C.c_double, _DP]
        L.ref_geodesic_observables.argtypes = [_DP, C.c_double, C.c_double, _DP]
        L.ref_locate_cell.argtypes = [C.c_size_t] * 3 + [_DP] * 3 + [C.c_double] * 3 + [C.POINTER(C.c_int)]
        L.ref_parse_output_variables.argtypes = [C.c_char_p, C.POINTER(C.c_int32), C.POINTER(C.c_size_t)]

    @staticmethod
    def available():
        return REF_SO.exists()

    @staticmethod
    def root():
        """The reference project's root directory oracle/_ref was built from,
        when that tree is present on this machine (else None)."""
        f = REF_SO.parent / "reference_root.txt"
        try:
            root = Path(f.read_text().strip())
        except OSError:
            return None
        return root if root.is_dir() else None

    def error(self):
        return self.lib.ref_last_error().decode()

    def parse_output_variables(self, spec: str):
        """The reference's OutputSelection::parse: field indices in write order."""
        fields = (C.c_int32 * 40)()
        count = C.c_size_t(0)
        if self.lib.ref_parse_output_variables(spec.encode(), fields, C.byref(count)) != 0:
            raise ValueError(self.error())
        return [fields[k] for k in range(count.value)]

    def params_from_toml(self, path) -> Params:
        p = Params()
        if self.lib.ref_params_from_toml(str(path).encode(), C.byref(p)) != 0:
            raise ValueError(self.error())
        return p

    def adapter_params_from_toml(self, path) -> Params:
        """grt_params as the product's drop-in adapter maps the structs the
        reference's own loader fills from this config."""
        p = Params()
        if self.lib.ref_adapter_params_from_toml(str(path).encode(), C.byref(p)) != 0:
            raise ValueError(self.error())
        return p

    def init_image_photons(self, toml, nx, ny, id_offset=0) -> PhotonArrays:
        ph = PhotonArrays(nx * ny)
        soa = ph.soa()
        if self.lib.ref_init_image_photons(str(toml).encode(), nx, ny, id_offset, C.byref(soa)) != 0:
            raise ValueError(self.error())
        return ph

    def init_image_photons_random(self, toml, n, id_offset=0) -> PhotonArrays:
        """The reference's own initialize_photons_image, random screen and all."""
        ph = PhotonArrays(n)
        soa = ph.soa()
        if self.lib.ref_init_image_photons_random(str(toml).encode(), n, id_offset, C.byref(soa)) != 0:
            raise ValueError(self.error())
        return ph

    def init_disk_photons(self, toml, numpy_dir=None, id_offset=0) -> PhotonArrays:
        """The reference's own disk-mode emission (its cell offsets and initialiser)."""
        nd = str(numpy_dir).encode() if numpy_dir else None
        n = C.c_uint64(0)
        if self.lib.ref_init_disk_photons(str(toml).encode(), nd, id_offset, None, C.byref(n)) != 0:
            raise ValueError(self.error())
        ph = PhotonArrays(n.value)
        soa = ph.soa()
        if self.lib.ref_init_disk_photons(str(toml).encode(), nd, id_offset, C.byref(soa), C.byref(n)) != 0:
            raise ValueError(self.error())
        return ph

    def run(self, toml, photons: PhotonArrays, p: Params = None, numpy_dir=None, output_dir=None):
        """Run the reference's integrate_geodesics in place; returns (products|None, stats)."""
        prod = ProductArrays.for_params(p) if p is not None else None
        ps = prod.struct() if prod is not None else None
        elapsed = C.c_double(0.0)
        stepped = C.c_uint64(0)
        live = C.c_uint64(0)
        soa = photons.soa()
        rc = self.lib.ref_run_photons(str(toml).encode(), numpy_dir.encode() if numpy_dir else None,
                                      str(output_dir).encode() if output_dir else None, C.byref(soa),
                                      photons.n, C.byref(ps) if ps is not None else None,
                                      C.byref(elapsed), C.byref(stepped), C.byref(live))
        if rc != 0:
            raise RuntimeError(self.error())
        return prod, {"elapsed_s": elapsed.value, "stepped": stepped.value, "live_calls": live.value}

    def rhs(self, X, P, a, M):
        out = np.zeros(8)
        self.lib.ref_hamiltonian_rhs(_dp(np.asarray(X, float)), _dp(np.asarray(P, float)), a, M, _dp(out))
        return out

    def null_momentum(self, X, K, a, M):
        out = np.zeros(4)
        ok = self.lib.ref_null_momentum(_dp(np.asarray(X, float)), _dp(np.asarray(K, float)), a, M, _dp(out))
        return bool(ok), out

    def observables(self, state, a, M):
        out = np.zeros(4)
        self.lib.ref_geodesic_observables(_dp(np.asarray(state, float)), a, M, _dp(out))
        return out

    def locate_cell(self, r, th, ph, radius, polar, azimuth):
        r = np.ascontiguousarray(r, float); th = np.ascontiguousarray(th, float); ph = np.ascontiguousarray(ph, float)
        ijk = (C.c_int * 3)()
        ok = self.lib.ref_locate_cell(*r.shape, _dp(r), _dp(th), _dp(ph), radius, polar, azimuth, ijk)
        return bool(ok), tuple(ijk)


def compare_photons(a: PhotonArrays, b: PhotonArrays, rtol=1e-9):
    """Per-field max relative difference between two photon SoAs (floats) and
    exact mismatch counts (integers)."""
    out = {}
    for f in ("id", "terminate", "phase"):
        out[f] = int(np.count_nonzero(getattr(a, f) != getattr(b, f)))
    for f in ("frequency", "emission_frame_energy", "x0", "x1", "x2", "x3", "k0", "k1", "k2", "k3",
              "I", "Q", "U", "V", "dlambda", "theta_disp", "phi_disp"):
        x, y = getattr(a, f), getattr(b, f)
        scale = np.maximum(np.maximum(np.abs(x), np.abs(y)), 1e-300)
        d = np.abs(x - y) / scale
        d[(x == y)] = 0.0
        out[f] = float(np.max(d)) if d.size else 0.0
    return out
