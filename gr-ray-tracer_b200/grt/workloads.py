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

from .abi import GEN_CUSTOM, MODE_IMAGE, PREC_FP64, RK4, RK45, Params
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

WORKLOADS = {"c1": C1, "c2": C2}


def scaled(w: ImageWorkload, pixels=None, grid=None, **extra) -> ImageWorkload:
    """A smaller copy of a workload for parity tests (same physics, fewer rays/cells)."""
    return ImageWorkload(w.name + "_small", grid or w.grid, w.spin, w.inclination_deg,
                         pixels or w.pixels, w.integrator, w.initial_step, w.max_steps, w.rtol,
                         w.atol, w.kappa, w.jcoef, w.precision, dict(w.extra, **extra))
