"""Standard-atmosphere profiles (drop-in for ``pylblrtm/profiles.py:108-172``).

The tables are public standard data (US Standard Atmosphere 1976 pressure and
temperature; AFGL mid-latitude-summer mixing ratios, CO2 at 415 ppm). They must
hold the same numbers as the reference tables (``profiles.py:27-98``) for the
standard profile to produce the same layers.
"""

from __future__ import annotations

from typing import Dict, List, Optional

import numpy as np

from .atmosphere import AtmosphericProfile

# Altitude-ascending tables; reversed to top-of-atmosphere first on output.
USSA_ALT_KM = np.array([0., 1., 2., 3., 4., 5., 6., 7., 8., 9., 10., 11.,
                        12., 15., 20., 25., 30., 35., 40., 45., 50.])
USSA_P_HPA = np.array([1013.25, 898.76, 794.95, 701.09, 616.40, 540.48, 471.81, 410.61,
                       356.00, 307.42, 264.36, 226.32, 193.99, 121.12, 55.293, 25.492,
                       11.970, 5.7459, 2.8714, 1.4910, 0.79779])
USSA_T_K = np.array([288.15, 281.65, 275.15, 268.66, 262.17, 255.68, 249.19, 242.70,
                     236.22, 229.73, 223.25, 216.65, 216.65, 216.65, 216.65, 221.55,
                     226.51, 236.51, 250.35, 264.16, 270.65])

VMR_ALT_KM = np.array([0., 1., 2., 3., 4., 5., 7., 10., 12., 15., 20., 25., 30., 35., 40., 45., 50.])
_GAS_TABLES: Dict[str, np.ndarray] = {
    "H2O": np.array([7.745e-3, 5.200e-3, 3.150e-3, 1.845e-3, 1.017e-3, 5.630e-4,
                     1.300e-4, 3.000e-5, 9.000e-6, 3.500e-6, 2.900e-6, 3.200e-6,
                     3.300e-6, 3.300e-6, 3.300e-6, 3.300e-6, 3.300e-6]),
    "CO2": np.full(VMR_ALT_KM.size, 415.0e-6),
    "O3": np.array([2.0e-8, 2.5e-8, 2.8e-8, 3.0e-8, 4.0e-8, 7.0e-8,
                    1.2e-7, 1.8e-7, 2.6e-7, 8.0e-7, 5.0e-6, 8.0e-6,
                    7.5e-6, 5.7e-6, 3.0e-6, 1.1e-6, 4.2e-7]),
    "N2O": np.array([3.20e-7, 3.20e-7, 3.20e-7, 3.20e-7, 3.20e-7, 3.20e-7,
                     3.20e-7, 3.20e-7, 3.15e-7, 3.10e-7, 2.80e-7, 2.20e-7,
                     1.50e-7, 7.50e-8, 2.50e-8, 6.00e-9, 1.00e-9]),
    "CH4": np.array([1.800e-6, 1.800e-6, 1.800e-6, 1.800e-6, 1.800e-6, 1.800e-6,
                     1.800e-6, 1.790e-6, 1.770e-6, 1.760e-6, 1.600e-6, 1.200e-6,
                     7.500e-7, 3.500e-7, 1.700e-7, 7.000e-8, 3.000e-8]),
    "CO": np.array([1.50e-7, 1.20e-7, 1.00e-7, 8.0e-8, 7.0e-8, 6.0e-8,
                    5.0e-8, 4.5e-8, 4.5e-8, 5.0e-8, 5.0e-8, 4.5e-8,
                    5.0e-8, 6.5e-8, 9.5e-8, 1.45e-7, 2.00e-7]),
}


def log_vmr_interp(z_query: np.ndarray, gas: str) -> np.ndarray:
    """Mixing ratio at altitudes ``z_query`` [km], linear in log(VMR), clamped."""
    table = _GAS_TABLES[gas]
    return np.exp(np.interp(z_query, VMR_ALT_KM, np.log(np.clip(table, 1e-30, None))))


def us_standard_atmosphere(gases: Optional[List[str]] = None,
                           alt_max_km: float = 50.0) -> AtmosphericProfile:
    """USSA76 levels up to ``alt_max_km`` with AFGL MLS mixing ratios, TOA first."""
    available = list(_GAS_TABLES.keys())
    if gases is None:
        gases = available
    else:
        unknown = [g for g in gases if g not in _GAS_TABLES]
        if unknown:
            raise ValueError(f"Unknown gas(es): {unknown}. Available: {available}")
    if alt_max_km > 50.0:
        raise ValueError("alt_max_km must be ≤ 50 km (USSA table limit)")
    keep = USSA_ALT_KM <= alt_max_km + 1e-6
    alt = USSA_ALT_KM[keep]
    vmr = {g: log_vmr_interp(alt, g) for g in gases}
    return AtmosphericProfile(
        pressure_hpa=USSA_P_HPA[keep][::-1].copy(),
        temperature_k=USSA_T_K[keep][::-1].copy(),
        vmr={g: v[::-1].copy() for g, v in vmr.items()},
    )


def list_profile_gases() -> List[str]:
    """Gas names the standard profile library provides."""
    return list(_GAS_TABLES.keys())
