"""Atmospheric levels and hydrostatic layers (drop-in for ``pylblrtm/atmosphere.py``).

``AtmosphericProfile`` validates levels exactly like ``atmosphere.py:63-100``.
``build_layers`` is kept on the host for API compatibility
(``atmosphere.py:110-141``); the forward engine builds the same layers on the
device (``lbl_build_layers``) with the same operation order, and the tests check
the two agree bit for bit.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Dict

import numpy as np

AVOGADRO = 6.02214086e23     # mol^-1
GRAVITY = 9.80665            # m s^-2
M_DRY_AIR = 0.0289644        # kg mol^-1
P_STD_HPA = 1013.25          # hPa
# molecules per m^2 per Pa of pressure difference; evaluated in the same order
# as atmosphere.py:134 so host and device use the identical double.
COLUMN_FACTOR = AVOGADRO / (GRAVITY * M_DRY_AIR)


@dataclass
class _Layers:
    """Layer means, index 0 = topmost layer; all arrays shape (n_layers,)."""

    pressure_atm: np.ndarray
    temperature_k: np.ndarray
    vmr: Dict[str, np.ndarray]
    column_cm2: Dict[str, np.ndarray]

    @property
    def n_layers(self) -> int:
        return len(self.pressure_atm)


class AtmosphericProfile:
    """Levels ordered top of atmosphere first (pressure strictly increasing)."""

    def __init__(self, pressure_hpa, temperature_k, vmr: Dict[str, object]) -> None:
        p = np.asarray(pressure_hpa, dtype=np.float64)
        t = np.asarray(temperature_k, dtype=np.float64)
        if p.ndim != 1 or p.size < 2:
            raise ValueError("pressure_hpa must be a 1-D array with at least 2 levels")
        if not np.all(np.isfinite(p)) or np.any(p <= 0):
            raise ValueError("pressure_hpa must be finite and positive")
        if np.any(np.diff(p) <= 0):
            raise ValueError(
                "pressure_hpa must be strictly increasing from TOA "
                "(smallest pressure = highest altitude = index 0)"
            )
        if t.shape != p.shape:
            raise ValueError("temperature_k must have the same length as pressure_hpa")
        if not np.all(np.isfinite(t)) or np.any(t <= 0):
            raise ValueError("temperature_k must be finite and positive")
        clean: Dict[str, np.ndarray] = {}
        for gas, values in vmr.items():
            v = np.asarray(values, dtype=np.float64)
            if v.shape != p.shape:
                raise ValueError(
                    f"vmr['{gas}'] must have the same length as pressure_hpa "
                    f"({p.size}), got {v.size}"
                )
            if not np.all(np.isfinite(v)) or np.any(v < 0) or np.any(v > 1):
                raise ValueError(f"vmr['{gas}'] must be finite and in [0, 1]")
            clean[gas] = v
        self.pressure_hpa = p
        self.temperature_k = t
        self.vmr = clean

    @property
    def n_levels(self) -> int:
        return self.pressure_hpa.size

    @property
    def n_layers(self) -> int:
        return self.n_levels - 1

    def build_layers(self) -> _Layers:
        """Geometric-mean pressure, arithmetic-mean T and VMR, hydrostatic columns."""
        p = self.pressure_hpa
        t = self.temperature_k
        p_layer = np.sqrt(p[:-1] * p[1:]) / P_STD_HPA
        t_layer = 0.5 * (t[:-1] + t[1:])
        vmr_layer = {gas: 0.5 * (v[:-1] + v[1:]) for gas, v in self.vmr.items()}
        air_col = COLUMN_FACTOR * (np.abs(np.diff(p)) * 100.0) / 1e4
        col = {gas: v * air_col for gas, v in vmr_layer.items()}
        return _Layers(p_layer, t_layer, vmr_layer, col)

    def __repr__(self) -> str:
        return (
            f"AtmosphericProfile({self.n_levels} levels, "
            f"P=[{self.pressure_hpa[0]:.4g}–{self.pressure_hpa[-1]:.4g}] hPa, "
            f"T=[{self.temperature_k.min():.1f}–{self.temperature_k.max():.1f}] K, "
            f"gases={list(self.vmr.keys())})"
        )
