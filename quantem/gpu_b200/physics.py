"""Electron wavelength for the SSB calibration.

Restates ``wavelength_A_from_kV`` / ``electron_wavelength_angstrom`` of the
reference (bobleesj/quantem.gpu ``src/quantem/gpu/optics/physics.py:33-86,
177-200``): table values for the common integral voltages (so 300 kV gives
0.019687489006849 A exactly), otherwise the relativistic de Broglie formula.
"""
from __future__ import annotations

import math

PLANCK_H = 6.62607015e-34
ELECTRON_MASS = 9.1093837015e-31
ELECTRON_CHARGE = 1.602176634e-19
SPEED_OF_LIGHT = 299792458.0

COMMON_VOLTAGES_A = {
    80: 0.041757160772834,
    120: 0.033492152726724,
    200: 0.025079340450548,
    300: 0.019687489006849,
    400: 0.016439434169908,
}


def wavelength_angstrom(voltage_kV: float) -> float:
    """Relativistic electron wavelength (Angstrom) at ``voltage_kV``."""
    v_int = int(voltage_kV)
    if v_int == voltage_kV and v_int in COMMON_VOLTAGES_A:
        return COMMON_VOLTAGES_A[v_int]
    volts = voltage_kV * 1e3
    gamma = 1.0 + ELECTRON_CHARGE * volts / (2.0 * ELECTRON_MASS * SPEED_OF_LIGHT ** 2)
    lam_m = PLANCK_H / math.sqrt(2.0 * ELECTRON_MASS * ELECTRON_CHARGE * volts * gamma)
    return lam_m * 1e10


def electron_wavelength_angstrom(energy_ev: float) -> float:
    """Wavelength (Angstrom) for an electron energy in eV."""
    return wavelength_angstrom(energy_ev / 1000.0)
