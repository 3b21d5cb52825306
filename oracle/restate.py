"""Float64 restatement of the reference forward model — TEST INFRASTRUCTURE ONLY.

Every function cites the reference lines it follows. Inputs are plain arrays
and dicts (no package objects), so the oracle stays independent of the code it
checks. The Voigt profile uses ``scipy.special.wofz`` exactly like the
reference (``pylblrtm/forward.py:22,51-62``); scipy is the third-party
dependency holding the Faddeeva algorithm (pinned only as ``scipy>=1.10`` in
``pyproject.toml:15``; 1.18.1 in this image).

Parity status: pinned — ``tests/test_oracle.py`` checks these functions against
golden vectors generated by running the reference (``tests/golden/``).
"""

from __future__ import annotations

import math
import warnings
from typing import Dict, Tuple

import numpy as np
from scipy.special import wofz

T_REF = 296.0                          # forward.py:32
C2 = 1.4387752                         # forward.py:33
DOPPLER = 3.5810e-7                    # forward.py:34
SQRT_LN2 = math.sqrt(math.log(2.0))    # forward.py:35
VOIGT_K = SQRT_LN2 / math.sqrt(math.pi)  # forward.py:36

AVOGADRO = 6.02214086e23               # atmosphere.py:15
GRAVITY = 9.80665                      # atmosphere.py:16
M_DRY_AIR = 0.0289644                  # atmosphere.py:17
P_STD_HPA = 1013.25                    # atmosphere.py:18

# HITRAN global molecule numbers (hitran_manager.py:89-101), id -> name.
_MOL_NAMES = dict(enumerate(
    ["H2O", "CO2", "O3", "N2O", "CO", "CH4", "O2", "NO", "SO2", "NO2", "NH3", "HNO3",
     "OH", "HF", "HCl", "HBr", "HI", "ClO", "OCS", "H2CO", "HOCl", "N2", "HCN", "CH3Cl",
     "H2O2", "C2H2", "C2H6", "PH3", "COF2", "SF6", "H2S", "HCOOH", "HO2", "O", "ClONO2",
     "NO+", "HOBr", "C2H4", "CH3OH", "CH3Br", "CH3CN", "CF4", "C4H2", "HC3N", "H2", "CS",
     "SO3", "C2N2", "COCl2"], start=1))
_MOL_NAMES.update({51: "SO", 52: "CH3F", 53: "GeH4", 54: "CS2", 55: "CH3I", 56: "NF3"})


def grid(nu_min: float, nu_max: float, step: float) -> np.ndarray:
    """Uniform grid, forward.py:141-142."""
    n_pts = int(np.ceil((nu_max - nu_min) / step)) + 1
    return nu_min + np.arange(n_pts, dtype=np.float64) * step


def build_layers(p_hpa, t_k, vmr: Dict[str, np.ndarray]):
    """Hydrostatic layers, atmosphere.py:117-141. Returns (p_atm, T, vmr_layer, col)."""
    p = np.asarray(p_hpa, dtype=np.float64)
    t = np.asarray(t_k, dtype=np.float64)
    p_layer = np.sqrt(p[:-1] * p[1:]) / P_STD_HPA
    t_layer = 0.5 * (t[:-1] + t[1:])
    vmr_layer = {g: 0.5 * (np.asarray(v)[:-1] + np.asarray(v)[1:]) for g, v in vmr.items()}
    dp_pa = np.abs(np.diff(p)) * 100.0
    col_factor = AVOGADRO / (GRAVITY * M_DRY_AIR)
    air_col = col_factor * dp_pa / 1e4
    col = {g: v * air_col for g, v in vmr_layer.items()}
    return p_layer, t_layer, vmr_layer, col


def q_interp(T: float, t_arr: np.ndarray, q_arr: np.ndarray) -> float:
    """Partition sum by clamped linear interpolation, spectral_data.py:43-52."""
    return float(np.interp(T, t_arr, q_arr))


def radiation_term(nu, T: float):
    """JRAD=0 radiation term nu*tanh(c2*nu/2T), forward.py:41-48."""
    return nu * np.tanh(0.5 * C2 * nu / T)


def voigt(nu, centers, doppler, lorentz):
    """Voigt matrix [n_nu x n_lines], forward.py:51-62."""
    z = SQRT_LN2 * ((nu[:, None] - centers) + 1j * lorentz) / doppler
    return wofz(z).real * (VOIGT_K / doppler)


def prepare_groups(nu, lines, tips, masses, profile_gases, p_atm, t_layer, cutoff):
    """Group selection, masks, molar masses and Q ratios, forward.py:189-245."""
    nu0 = lines["nu0"]
    delta = lines["shift"]
    mol_ids = lines["mol_id"]
    iso_ids = lines["iso_id"]
    max_p = float(p_atm.max()) if p_atm.size > 0 else 1.0
    shift_bound = np.abs(delta) * max_p
    pairs = sorted(set(zip(mol_ids.tolist(), iso_ids.tolist())))
    prepared = []
    for mol_id, iso_id in pairs:
        gas = _MOL_NAMES.get(int(mol_id))
        if gas is None:
            warnings.warn(f"mol_id={mol_id} is not in the HITRAN catalogue; lines skipped.",
                          RuntimeWarning, stacklevel=3)
            continue
        if gas not in profile_gases:
            warnings.warn(
                f"Gas '{gas}' (mol_id={mol_id}, iso_id={iso_id}) is in the "
                f"spectral data but not in the atmospheric profile vmr; "
                f"its lines are skipped.", RuntimeWarning, stacklevel=3)
            continue
        mask = ((mol_ids == mol_id) & (iso_ids == iso_id)
                & (nu0 >= nu[0] - cutoff - shift_bound)
                & (nu0 <= nu[-1] + cutoff + shift_bound))
        if not mask.any():
            continue
        key = (int(mol_id), int(iso_id))
        mm = masses.get(key)
        if mm is None:
            warnings.warn(f"No molar mass found for (mol_id={mol_id}, iso_id={iso_id}); "
                          f"using dry-air mass as fallback.", RuntimeWarning, stacklevel=3)
            mm = 28.97
        if key not in tips:
            raise KeyError(f"No TIPS data for (mol_id={mol_id}, iso_id={iso_id}). "
                           f"Available: {sorted(tips.keys())}")
        t_arr, q_arr = tips[key]
        q_ref = q_interp(T_REF, t_arr, q_arr)
        q_ratios = np.array([q_ref / q_interp(float(T), t_arr, q_arr) for T in t_layer])
        prepared.append((mol_id, iso_id, gas, mask, mm, q_ratios))
    return prepared


def line_params(k, lines, p_atm, t_layer, vmr_layer, col, grp):
    """Per-layer line quantities for one group, forward.py:249-292.

    Returns (idx, shifted, strength, lorentz, doppler) or None when col == 0.
    """
    _, _, gas, mask, mm, q_ratios = grp
    T = float(t_layer[k])
    P = float(p_atm[k])
    c = float(col[gas][k])
    if c == 0.0:
        return None
    vmr_gas = float(vmr_layer[gas][k])
    p_self = vmr_gas * P
    p_air = P - p_self
    idx = np.flatnonzero(mask)
    centers = lines["nu0"][idx]
    shifted = centers + lines["shift"][idx] * p_air
    strength = (lines["Sref"][idx] * q_ratios[k]
                * np.exp(-C2 * lines["Elow"][idx] * (1.0 / T - 1.0 / T_REF))
                * (-np.expm1(-C2 * centers / T))
                / (-np.expm1(-C2 * centers / T_REF))
                * c / radiation_term(shifted, T))
    if not np.isfinite(strength).all() or np.any(strength < 0):
        raise FloatingPointError(f"Layer {k}, gas '{gas}': non-finite or negative line strength")
    lorentz = (T_REF / T) ** lines["n_air"][idx] * (lines["g_air"][idx] * p_air
                                                    + lines["g_self"][idx] * p_self)
    doppler = centers * DOPPLER * math.sqrt(T / mm)
    return idx, shifted, strength, lorentz, doppler


def optical_depth(nu, lines, tips, masses, p_atm, t_layer, vmr_layer, col,
                  cutoff=25.0, tile_width=2.0):
    """Per-layer optical depth [n_layers, n_nu], forward.py:157-317."""
    n_layers = p_atm.size
    n_nu = nu.size
    od = np.zeros((n_layers, n_nu), dtype=np.float64)
    step = float(nu[1] - nu[0]) if n_nu > 1 else 0.001
    tile = max(1, int(np.floor(tile_width / step + 1e-8)))
    prepared = prepare_groups(nu, lines, tips, masses, tuple(col.keys()), p_atm, t_layer, cutoff)
    if not prepared:
        return od
    for k in range(n_layers):
        T = float(t_layer[k])
        for grp in prepared:
            lp = line_params(k, lines, p_atm, t_layer, vmr_layer, col, grp)
            if lp is None:
                continue
            _, shifted, strength, lorentz, doppler = lp
            for t0 in range(0, n_nu, tile):
                t1 = min(t0 + tile, n_nu)
                seg = nu[t0:t1]
                near = (shifted >= seg[0] - cutoff) & (shifted <= seg[-1] + cutoff)
                if not near.any():
                    continue
                nb = np.flatnonzero(near)
                for b0 in range(0, nb.size, 256):
                    b = nb[b0:b0 + 256]
                    od[k, t0:t1] += voigt(seg, shifted[b], doppler[b], lorentz[b]) @ strength[b]
        od[k] *= radiation_term(nu, T)
        if not np.isfinite(od[k]).all():
            raise FloatingPointError(f"Layer {k}: non-finite optical depth after radiation term")
    return od


def transmittance(nu, od, mu=1.0):
    """Column transmittance exp(-sum_k od / mu), forward.py:151."""
    return np.exp(-od.sum(axis=0) / mu)


def count_evals(nu, lines, tips, masses, p_atm, t_layer, vmr_layer, col, cutoff=25.0, tile_width=2.0):
    """Number of (layer, grid point, line) Voigt evaluations of forward.py:295-309.

    Counts the pairs admitted by the tile-window test, using sorted shifted
    centres and binary search per tile instead of the reference's masks.
    """
    n_nu = nu.size
    step = float(nu[1] - nu[0]) if n_nu > 1 else 0.001
    tile = max(1, int(np.floor(tile_width / step + 1e-8)))
    prepared = prepare_groups(nu, lines, tips, masses, tuple(col.keys()), p_atm, t_layer, cutoff)
    t0 = np.arange(0, n_nu, tile)
    t1 = np.minimum(t0 + tile, n_nu)
    lo = nu[t0] - cutoff
    hi = nu[t1 - 1] + cutoff
    total = 0
    for k in range(p_atm.size):
        for grp in prepared:
            lp = line_params(k, lines, p_atm, t_layer, vmr_layer, col, grp)
            if lp is None:
                continue
            s = np.sort(lp[1])
            cnt = np.searchsorted(s, hi, side="right") - np.searchsorted(s, lo, side="left")
            total += int(np.sum(np.maximum(cnt, 0) * (t1 - t0)))
    return total
