"""The benchmark workloads (synthetic Fishbone-Moncrief tori; no public dataset).

Each workload fixes the reference-config keys the benchmark statement leaves
open, in the reference's own units (M = 1):

  camera.distance = 1000 (so termination.r_max = 1.5 * 1000 = 1500 and the
  image rays start with dlambda = initial_step * 1000), camera.phi = 0, a
  +/-20 M field of view (width = height = 40), termination.r_min = r_horizon,
  photons.generator = "custom" (deterministic frequency), and
  superphoton_count_normalization = 1e7 so that every grid cell, including the
  rho = 1e-6 atmosphere, emits at least one packet (int(rho * norm) >= 1);
  with a smaller normalisation every ray that meets the atmosphere first is
  rejected and the image is empty.  termination_percent = 1 and a large
  output.interval make the run end when every ray has terminated.

Rays are one per pixel centre (the deterministic pixel grid of
grt_init_image_photons) instead of the reference's random screen draw.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

from .abi import GEN_BLACKBODY, GEN_CUSTOM, MODE_DISK, MODE_IMAGE, PREC_FP64, RK4, RK45, ImageSpec, Params
from .config import reference_defaults


@dataclass
class ImageWorkload:
    name: str
    grid: tuple
    spin: float
    inclination_deg: float
    pixels: int
    integrator: int
    initial_step: float
    max_steps: int
    rtol: float = 1e-8
    atol: float = 1e-8
    kappa: float = 1.0
    jcoef: float = 1.0
    precision: int = PREC_FP64
    extra: dict = field(default_factory=dict)

    def params(self) -> Params:
        p = reference_defaults()
        horizon = 1.0 + math.sqrt(max(0.0, 1.0 - self.spin * self.spin))
        p.update(mode=MODE_IMAGE, integrator=self.integrator, precision=self.precision,
                 generator=GEN_CUSTOM, mass=1.0, spin=self.spin,
                 camera_distance=1000.0, camera_theta=math.radians(self.inclination_deg),
                 camera_phi=0.0, camera_width=40.0, camera_height=40.0,
                 r_term_min=horizon, r_term_max=1500.0, atol=self.atol, rtol=self.rtol,
                 max_steps=self.max_steps, termination_percent=1.0, output_interval=10**9,
                 nphotons=self.pixels * self.pixels, initial_step=self.initial_step,
                 absorption_enabled=1, emission_enabled=1,
                 absorption_coefficient=self.kappa, emission_coefficient=self.jcoef,
                 scattering_enabled=0, superphoton_count_normalization=1.0e7,
                 energy_per_cell_erg=1.0, custom_frequency_hz=2.30e11,
                 image_nx=self.pixels, image_ny=self.pixels, spectrum_bins=128,
                 spectrum_min_hz=1.0e8, spectrum_max_hz=1.0e22)
        p.update(**self.extra)
        return p

    def torus(self):
        from .torus import benchmark_torus
        return benchmark_torus(*self.grid, spin=self.spin)


# Plain FP64 image mode, RK4 fixed step (dlambda = 2 M), 64x64 px, 64x32x32 grid, a = 0.9, 60 deg.
C1 = ImageWorkload("c1_rk4_64px", (64, 32, 32), 0.9, 60.0, 64, RK4, 0.002, 1200)
# RK45 rtol = atol = 1e-8, 256x256 px, 128x64x64 grid, a = 0.94, 17 deg.
C2 = ImageWorkload("c2_rk45_256px", (128, 64, 64), 0.94, 17.0, 256, RK45, 0.01, 4000)

# Frequency channels of a batch: custom generator frequency f and an emission
# coefficient scaled by f / 230 GHz.
FREQ_CHANNELS_GHZ = (230.0, 345.0, 86.0, 43.0)


@dataclass
class BatchWorkload:
    """Several images traced by one persistent launch (grt_init_image_batch):
    each entry is (inclination_deg, pixels, frequency_ghz)."""
    name: str
    base: ImageWorkload
    images: list

    def params(self) -> Params:
        return self.base.params()

    def specs(self, p: Params | None = None) -> list:
        p = p or self.params()
        out = []
        for incl, px, f_ghz in self.images:
            out.append(ImageSpec.from_params(p, px, px, camera_theta=math.radians(incl),
                                             custom_frequency_hz=f_ghz * 1e9,
                                             emission_coefficient=p.emission_coefficient * f_ghz / 230.0))
        return out

    @property
    def rays(self) -> int:
        return sum(px * px for _, px, _ in self.images)

    def torus(self):
        return self.base.torus()


def _c3_images(seed=3):
    import numpy as np
    rng = np.random.default_rng(seed)
    incl = np.linspace(5.0, 85.0, 16)
    sizes = (64, 128, 256, 512)
    return [(float(i), int(sizes[rng.integers(0, 4)]), f) for i in incl for f in FREQ_CHANNELS_GHZ]


# The 256x256 RK45 image of C2 at the four frequency channels, one launch.
C2_BATCH = BatchWorkload("c2_rk45_256px_x4freq", C2, [(C2.inclination_deg, C2.pixels, f) for f in FREQ_CHANNELS_GHZ])
# 16 inclinations (5..85 deg) x 4 frequency channels, image sizes drawn from
# {64,128,256,512}^2 (seeded), RK45 over a 128x64x64 torus with a = 0.9.
C3 = BatchWorkload("c3_batch_64img", ImageWorkload("c3_base", (128, 64, 64), 0.9, 60.0, 256, RK45, 0.01, 4000),
                   _c3_images())

# Adjoint: 128x128 Stokes-I image, 96x48x48 torus, a = 0.9, 60 deg, RK45,
# checkpoints every 64 calls.  The image is made of line-of-sight forward rays
# (grt_init_image_forward_photons): the reference's own image mode emits at
# the first fluid contact and retraces its path outward, so its forward leg
# samples no fluid and the image does not depend on the multipliers at all.
# Forward rays start C4_BACK_DISTANCE behind the scene, cross the torus and
# are binned where they cross the camera plane, here at 100 M with a +/-30 M
# window so that lensed rays still land on it.
C4 = ImageWorkload("c4_adjoint_128px", (96, 48, 48), 0.9, 60.0, 128, RK45, 0.01, 4000,
                   extra=dict(camera_distance=100.0, camera_width=60.0, camera_height=60.0, r_term_max=150.0))
C4_CHECKPOINT_INTERVAL = 64
C4_BACK_DISTANCE = 60.0


def c4_target_multipliers(shape, seed=4, sigma=0.1):
    """Seeded lognormal multiplier fields exp(N(0, sigma)) for the target image."""
    import numpy as np
    rng = np.random.default_rng(seed)
    return np.exp(rng.normal(0.0, sigma, shape)), np.exp(rng.normal(0.0, sigma, shape))


@dataclass
class DiskWorkload:
    """Disk-mode scattering Monte Carlo (grt_init_disk_photons): packets from
    every torus cell, RK45, elastic (albedo 1) isotropic scattering in the
    fluid frame, absorption and emission on.  The Thomson optical depth across
    the torus is ~1 through the unit scales (scattering.optical_depth is not
    read by the reference): tau = sigma_T / m_p * rho_code * density_scale *
    path_code * length_scale ~ 0.4 * 0.5 * 0.5 * 10 = 1 for a 10 M chord at
    rho_code ~ 0.5.  Escape is termination beyond r_term_max."""
    name: str
    grid: tuple
    spin: float
    normalization: float
    r_escape: float = 100.0
    rtol: float = 1e-8
    initial_step: float = 0.01
    max_steps: int = 20000
    kappa: float = 0.1
    jcoef: float = 1e-10

    def params(self) -> Params:
        p = reference_defaults()
        horizon = 1.0 + math.sqrt(max(0.0, 1.0 - self.spin * self.spin))
        p.update(mode=MODE_DISK, integrator=RK45, precision=PREC_FP64, generator=GEN_BLACKBODY,
                 mass=1.0, spin=self.spin, r_term_min=horizon, r_term_max=self.r_escape,
                 atol=self.rtol, rtol=self.rtol, max_steps=self.max_steps, termination_percent=1.0,
                 output_interval=10**9, initial_step=self.initial_step,
                 absorption_enabled=1, emission_enabled=1, absorption_coefficient=self.kappa,
                 emission_coefficient=self.jcoef, scattering_enabled=1, scattering_albedo=1.0,
                 scattering_seed=2024, superphoton_count_normalization=self.normalization,
                 energy_per_cell_erg=1.0, density_g_cm3_per_code=0.5, length_cm_per_code=1.0,
                 temperature_k_per_code=1e11, camera_distance=self.r_escape)
        return p

    def torus(self):
        from .torus import benchmark_torus
        return benchmark_torus(*self.grid, spin=self.spin)


# 1e7 packets (normalisation 210 on the 128x64x64 torus: sum of int(rho * 210)
# over the cells), a = 0.9.
C5 = DiskWorkload("c5_disk_1e7", (128, 64, 64), 0.9, 210.0)


# single-image workload of each key (for c3, the batch's base image: 256x256 at 60 deg)
WORKLOADS = {"c1": C1, "c2": C2, "c3": C3.base}
# the C1 image at the four frequency channels (for the batched forms of --workload c1)
C1_BATCH = BatchWorkload("c1_rk4_64px_x4freq", C1, [(C1.inclination_deg, C1.pixels, f) for f in FREQ_CHANNELS_GHZ])
BATCHES = {"c1": C1_BATCH, "c2": C2_BATCH, "c3": C3}


def scaled(w: ImageWorkload, pixels=None, grid=None, **extra) -> ImageWorkload:
    """A smaller copy of a workload for parity tests (same physics, fewer rays/cells)."""
    return ImageWorkload(w.name + "_small", grid or w.grid, w.spin, w.inclination_deg,
                         pixels or w.pixels, w.integrator, w.initial_step, w.max_steps, w.rtol,
                         w.atol, w.kappa, w.jcoef, w.precision, dict(w.extra, **extra))
