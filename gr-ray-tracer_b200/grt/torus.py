"""Fishbone-Moncrief torus inputs in the reference's NumPy grid format.

Produces the seven float64 arrays the reference loader reads
(src/input/load_python_arrays.hpp:27-62): r, theta, phi, rho, Tgas with shape
(nr, ntheta, nphi) and vel, mag with shape (nr, ntheta, nphi, 4).

The construction follows the reference generator
create_fishbone_moncrief_torus (src/create_example_data.py:102-281): an
analytic hydrostatic torus of constant specific angular momentum (Fishbone &
Moncrief 1976) around a Kerr hole, a polytrope with the peak density
normalised to one, and a zero-angular-momentum-observer atmosphere at
rho_floor outside it.  Two knobs the reference script hard-codes are
parameters here, because the benchmark workloads need them:

  * theta_edge  -- theta runs over [theta_edge, pi - theta_edge]
                   (the reference fixes 1e-3, create_example_data.py:167);
  * r_min_factor -- the default inner radius r_min_factor * r_horizon
                   (the reference fixes 1.2, create_example_data.py:157-158).

With theta_edge=1e-3 and r_min_factor=1.2 the arrays are bitwise identical to
the reference script's (checked in tests/test_torus.py against arrays the
reference script itself produced), so the floating-point evaluation order
below mirrors the script's wherever it affects rounding.
"""

from __future__ import annotations

from pathlib import Path

import numpy as np

FIELD_FILES = ("r.npy", "theta.npy", "phi.npy", "rho.npy", "Tgas.npy", "vel.npy", "mag.npy")


def _keplerian_l(r_hat, a_hat):
    """Specific angular momentum L/E of a prograde circular equatorial orbit at M=1
    (Bardeen, Press & Teukolsky 1972, eq. 2.12-2.13)."""
    return (r_hat**2 - 2.0 * a_hat * np.sqrt(r_hat) + a_hat**2) / (
        r_hat**1.5 - 2.0 * np.sqrt(r_hat) + a_hat
    )


def _bl_metric(r_hat, theta, a_hat):
    """(g_tt, g_tphi, g_phiphi) of Boyer-Lindquist Kerr at M=1."""
    sin2 = np.sin(theta) ** 2
    sigma = r_hat**2 + a_hat**2 * np.cos(theta) ** 2
    delta = r_hat**2 - 2.0 * r_hat + a_hat**2
    big_a = (r_hat**2 + a_hat**2) ** 2 - delta * a_hat**2 * sin2
    return -(1.0 - 2.0 * r_hat / sigma), -2.0 * r_hat * a_hat * sin2 / sigma, big_a * sin2 / sigma


def _rotating_velocity(r_hat, theta, a_hat, ell):
    """u^t, u^phi and covariant u_t of a flow with u^r = u^theta = 0 and -u_phi/u_t = ell."""
    g_tt, g_tp, g_pp = _bl_metric(r_hat, theta, a_hat)
    omega = -(g_tp + ell * g_tt) / (g_pp + ell * g_tp)
    norm = -(g_tt + 2.0 * omega * g_tp + omega**2 * g_pp)
    with np.errstate(invalid="ignore", divide="ignore"):
        u_t_up = 1.0 / np.sqrt(norm)
    return u_t_up, omega * u_t_up, u_t_up * (g_tt + omega * g_tp)


def fishbone_moncrief_torus(nr=64, ntheta=64, nphi=32, r_min=None, r_max=50.0, mass=1.0,
                            spin=0.9375, r_in=6.0, r_pressure_max=10.0, gamma=4.0 / 3.0,
                            rho_floor=1.0e-6, theta_edge=1.0e-3, r_min_factor=1.2):
    """Return a dict name -> float64 array (keys are the .npy file names)."""
    if min(nr, ntheta, nphi) < 2:
        raise ValueError("nr, ntheta, and nphi must each be at least 2")
    if mass <= 0.0:
        raise ValueError("mass must be positive")
    if abs(spin) > mass:
        raise ValueError("require |spin| <= mass")
    if gamma <= 1.0:
        raise ValueError("gamma must be greater than 1")
    if not (r_pressure_max > r_in > 0.0):
        raise ValueError("require 0 < r_in < r_pressure_max")
    if not (0.0 <= theta_edge < np.pi / 2):
        raise ValueError("theta_edge must be in [0, pi/2)")
    horizon = mass + np.sqrt(mass**2 - spin**2)
    if r_min is None:
        r_min = r_min_factor * horizon
    if r_min <= horizon or r_max <= r_min:
        raise ValueError(f"require horizon ({horizon:.6g}) < r_min < r_max")

    r1 = np.logspace(np.log10(r_min), np.log10(r_max), nr)
    th1 = np.linspace(theta_edge, np.pi - theta_edge, ntheta)
    ph1 = np.linspace(0.0, 2.0 * np.pi, nphi, endpoint=False)
    radius, polar, azimuth = np.meshgrid(r1, th1, ph1, indexing="ij")

    a_hat = spin / mass
    r_hat = radius / mass
    ell = _keplerian_l(r_pressure_max / mass, a_hat)
    u_t_up, u_phi_up, u_t_dn = _rotating_velocity(r_hat, polar, a_hat, ell)
    _, _, u_t_dn_in = _rotating_velocity(np.array(r_in / mass), np.array(np.pi / 2.0), a_hat, ell)

    with np.errstate(invalid="ignore", divide="ignore"):
        enthalpy = u_t_dn_in / u_t_dn
    inside = (r_hat >= r_in / mass) & np.isfinite(enthalpy) & (enthalpy >= 1.0)
    density = np.where(
        inside,
        np.power(np.clip((gamma - 1.0) / gamma * (enthalpy - 1.0), 0.0, None), 1.0 / (gamma - 1.0)),
        0.0)
    peak = density.max()
    if peak > 0.0:
        density /= peak
    temperature = np.where(inside, np.power(np.maximum(density, 1e-300), gamma - 1.0), 0.0)
    density = np.where(inside, density, rho_floor)
    temperature = np.where(inside, temperature, rho_floor)

    g_tt, g_tp, g_pp = _bl_metric(r_hat, polar, a_hat)
    omega_zamo = -g_tp / g_pp
    lapse_sq = g_tp**2 / g_pp - g_tt
    zamo_u_t = 1.0 / np.sqrt(np.clip(lapse_sq, 1e-300, None))
    velocity = np.zeros((nr, ntheta, nphi, 4), dtype=np.float64)
    velocity[..., 0] = np.where(inside, u_t_up, zamo_u_t)
    velocity[..., 3] = np.where(inside, u_phi_up, omega_zamo * zamo_u_t) / mass
    magnetic = np.zeros_like(velocity)
    arrays = {"r.npy": radius, "theta.npy": polar, "phi.npy": azimuth, "rho.npy": density,
              "Tgas.npy": temperature, "vel.npy": velocity, "mag.npy": magnetic}
    return {k: np.ascontiguousarray(v, dtype=np.float64) for k, v in arrays.items()}


def write_numpy_dir(arrays, directory):
    """Write the arrays as the seven .npy files of a reference input directory."""
    out = Path(directory)
    out.mkdir(parents=True, exist_ok=True)
    for name in FIELD_FILES:
        np.save(out / name, arrays[name])
    return out


def load_numpy_dir(directory):
    """Read a reference input directory back into a dict name -> array."""
    d = Path(directory)
    missing = [n for n in FIELD_FILES if not (d / n).is_file()]
    if missing:
        raise FileNotFoundError(f"NumPy directory '{d}' is missing required file(s): {', '.join(missing)}")
    return {n: np.load(d / n) for n in FIELD_FILES}


def benchmark_torus(nr, ntheta, nphi, spin):
    """The torus of the benchmark workloads: M=1, r_in=6, r_pmax=12, gamma=4/3,
    rho_floor=1e-6, r log-spaced from 1.05 r_horizon to 50, theta in (0.01, pi-0.01)."""
    return fishbone_moncrief_torus(nr, ntheta, nphi, r_max=50.0, mass=1.0, spin=spin, r_in=6.0,
                                   r_pressure_max=12.0, gamma=4.0 / 3.0, rho_floor=1.0e-6,
                                   theta_edge=0.01, r_min_factor=1.05)
