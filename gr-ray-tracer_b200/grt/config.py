"""Reference-format TOML configs for the hot path.

The reference reads exactly one flat TOML file (src/input/toml_config.hpp:40-77);
this module writes such files from a Params struct, so the same file drives the
reference code and this build.  Keys and their meaning are the reference's
(src/input/toml_config.hpp:137-236, README key list).
"""

from __future__ import annotations

import math
from pathlib import Path

from .abi import GEN_BLACKBODY, GEN_CUSTOM, GEN_POWER_LAW, MODE_DISK, Params, RK4

_GENERATOR_NAMES = {GEN_BLACKBODY: "blackbody", GEN_POWER_LAW: "power-law", GEN_CUSTOM: "custom"}


def reference_defaults() -> Params:
    """The reference's compiled-in defaults (src/utils.cpp:4-37,
    src/simulation_options.hpp:13-32, photon_generation.hpp:18-50)."""
    p = Params()
    p.mode = 0
    p.integrator = 1
    p.precision = 0
    p.generator = GEN_BLACKBODY
    p.mass, p.spin = 1.0, 1.0
    horizon = p.mass + math.sqrt(max(0.0, p.mass * p.mass - p.spin * p.spin))
    p.camera_theta = math.pi / 4.0
    p.camera_phi = math.pi / 4.0
    p.camera_width = p.camera_height = 20.0
    p.camera_distance = 10000.0
    p.r_term_min = horizon
    p.r_term_max = 1.5 * p.camera_distance
    p.atol = p.rtol = 1e-8
    p.min_step_scale, p.max_step_scale, p.safety = 0.01, 10.0, 0.9
    p.max_steps = 10000
    p.termination_percent = 0.9
    p.output_interval = 1
    p.nphotons = 20
    p.initial_step = 0.1
    p.absorption_enabled = p.emission_enabled = 0
    p.absorption_coefficient = p.emission_coefficient = 0.0
    p.scattering_enabled = 0
    p.rank = 0
    p.scattering_albedo = 1.0
    p.scattering_seed = 12345
    p.superphoton_count_normalization = 1.0
    p.energy_per_cell_erg = 1.0
    p.power_law_slope = 2.0
    p.nu_min_hz, p.nu_max_hz = 1.0e9, 1.0e20
    p.custom_frequency_hz = 2.30e11
    p.length_cm_per_code = p.time_s_per_code = p.density_g_cm3_per_code = 1.0
    p.temperature_k_per_code = p.four_velocity_cm_s_per_code = p.magnetic_gauss_per_code = 1.0
    p.image_nx = p.image_ny = 256
    p.spectrum_bins = 128
    p.spectrum_min_hz, p.spectrum_max_hz = 1.0e8, 1.0e22
    return p


def _fmt(x: float) -> str:
    return repr(float(x))


def _b(x) -> str:
    return "true" if x else "false"


def toml_text(p: Params, numpy_dir: str, output_dir: str = "./output", name: str = "grt") -> str:
    """Render p as a reference TOML file (every key explicit, so the reference's
    defaults never leak in)."""
    lines = [
        "[simulation]",
        f'mode = "{"disk" if p.mode == MODE_DISK else "image"}"',
        f'name = "{name}"',
        "[input]",
        "vacuum = false",
        f'numpy_dir = "{numpy_dir}"',
        "[black_hole]",
        f"mass = {_fmt(p.mass)}",
        f"spin = {_fmt(p.spin)}",
        "[camera]",
        f"theta = {_fmt(p.camera_theta)}",
        f"phi = {_fmt(p.camera_phi)}",
        f"width = {_fmt(p.camera_width)}",
        f"height = {_fmt(p.camera_height)}",
        f"distance = {_fmt(p.camera_distance)}",
        "[photons]",
        f"count = {int(max(1, p.nphotons))}",
        f'generator = "{_GENERATOR_NAMES[p.generator]}"',
        f"superphoton_count_normalization = {_fmt(p.superphoton_count_normalization)}",
        f"energy_per_cell_erg = {_fmt(p.energy_per_cell_erg)}",
        f"power_law_slope = {_fmt(p.power_law_slope)}",
        f"nu_min_hz = {_fmt(p.nu_min_hz)}",
        f"nu_max_hz = {_fmt(p.nu_max_hz)}",
        f"custom_frequency_hz = {_fmt(p.custom_frequency_hz)}",
        "[units]",
        f"length_cm_per_code = {_fmt(p.length_cm_per_code)}",
        f"time_s_per_code = {_fmt(p.time_s_per_code)}",
        f"density_g_cm3_per_code = {_fmt(p.density_g_cm3_per_code)}",
        f"temperature_k_per_code = {_fmt(p.temperature_k_per_code)}",
        f"four_velocity_cm_s_per_code = {_fmt(p.four_velocity_cm_s_per_code)}",
        f"magnetic_gauss_per_code = {_fmt(p.magnetic_gauss_per_code)}",
        "[parallel]",
        "decomposition = [1, 1, -1]",
        "[integration]",
        f'integrator = "{"rk4" if p.integrator == RK4 else "rk45"}"',
        f"max_steps = {int(p.max_steps)}",
        f"termination_percent = {_fmt(p.termination_percent)}",
        f"initial_step = {_fmt(p.initial_step)}",
        f"atol = {_fmt(p.atol)}",
        f"rtol = {_fmt(p.rtol)}",
        "[termination]",
        f"r_min = {_fmt(p.r_term_min)}",
        f"r_max = {_fmt(p.r_term_max)}",
        "[output]",
        f'directory = "{output_dir}"',
        f"interval = {int(p.output_interval)}",
        "stride = 1",
        'variables = ["id", "frequency", "x0", "x1", "x2", "x3", "k0", "k1", "k2", "k3", '
        '"I", "Q", "U", "V", "terminate", "phase"]',
        f"image_nx = {int(p.image_nx)}",
        f"image_ny = {int(p.image_ny)}",
        f"spectrum_bins = {int(p.spectrum_bins)}",
        f"spectrum_min_hz = {_fmt(p.spectrum_min_hz)}",
        f"spectrum_max_hz = {_fmt(p.spectrum_max_hz)}",
        "[scattering]",
        f"enabled = {_b(p.scattering_enabled)}",
        "optical_depth = 0.0",
        f"albedo = {_fmt(p.scattering_albedo)}",
        f"seed = {int(p.scattering_seed)}",
        "[radiative_transfer]",
        f"absorption_enabled = {_b(p.absorption_enabled)}",
        f"emission_enabled = {_b(p.emission_enabled)}",
        f"absorption_coefficient = {_fmt(p.absorption_coefficient)}",
        f"emission_coefficient = {_fmt(p.emission_coefficient)}",
    ]
    return "\n".join(lines) + "\n"


def write_toml(p: Params, path, numpy_dir, output_dir="./output", name="grt") -> Path:
    path = Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    path.write_text(toml_text(p, str(numpy_dir), str(output_dir), name))
    return path
