"""Electron-optics scalars, evaluated in float64 on the host.

Restates ``wide_angle_propagation/propagation.py:14-95`` with the physical
constants the reference takes from ``ase.units`` (propagation.py:6), i.e. ASE's
default CODATA-2014 set, hard-coded because ASE is not a dependency here.
"""
from __future__ import annotations

import math

HPLANCK = 6.626070040e-34   # J s
C_LIGHT = 299792458.0       # m / s
M_E = 9.10938356e-31        # kg
Q_E = 1.6021766208e-19      # C


def electron_rest_energy() -> float:
    """E0 = m_e c^2 / e in eV (propagation.py:14-21)."""
    return M_E * C_LIGHT ** 2 / Q_E


def relativistic_mass_correction(energy: float) -> float:
    """1 + eE/(m_e c^2) (propagation.py:24-26)."""
    return 1 + Q_E * energy / (M_E * C_LIGHT ** 2)


def energy2mass(energy: float) -> float:
    """Relativistic mass in kg (propagation.py:29-35)."""
    return relativistic_mass_correction(energy) * M_E


def energy2wavelength(energy: float) -> float:
    """Relativistic de Broglie wavelength in Angstrom (propagation.py:38-50)."""
    return (HPLANCK * C_LIGHT
            / math.sqrt(energy * (2 * M_E * C_LIGHT ** 2 / Q_E + energy))
            / Q_E * 1.0e10)


def energy2sigma(energy: float) -> float:
    """Interaction parameter in 1/(V*Angstrom) (propagation.py:53-63).

    In SI: sigma = 2 pi m e lambda / h^2, converted to 1/(V*A).
    """
    lam_m = energy2wavelength(energy) * 1e-10
    return 2 * math.pi * energy2mass(energy) * Q_E * lam_m / HPLANCK ** 2 * 1e-10


def refractive_index_coefficients(energy: float):
    """Coefficients of the cancellation-free n(V) - 1 used by the kernels.

    n^2 = ((E+V)^2 + 2 E0 (E+V)) / (2 E E0 + E^2)  (propagation.py:70-81), so
    n^2 - 1 = r = V (2E0 + 2E + V) / (E (2E0 + E)) and
    n - 1 = r / (sqrt(1 + r) + 1).
    Returns (a, inv_den) with r = V (a + V) * inv_den.
    """
    E0 = electron_rest_energy()
    return 2 * E0 + 2 * energy, 1.0 / (energy * (2 * E0 + energy))


def refractive_index_minus_one(v: float, energy: float) -> float:
    """n(V) - 1 without cancellation (float64 scalar)."""
    a, inv_den = refractive_index_coefficients(energy)
    r = v * (a + v) * inv_den
    return r / (math.sqrt(1 + r) + 1)
