"""Seeded synthetic line lists and profiles for tests and benchmarks.

No HITRAN data ships with this package, so the workloads are drawn from fixed
distributions (uniform line centres, log-uniform strengths, uniform widths) and
fixed seeds. Every generator is deterministic for a given seed.
"""

from __future__ import annotations

from typing import Dict, List, Sequence, Tuple

import numpy as np

from .atmosphere import AtmosphericProfile
from .profiles import USSA_ALT_KM, USSA_P_HPA, USSA_T_K, log_vmr_interp, us_standard_atmosphere
from .spectral_data import SpectralData

# (mol_id, molar mass g/mol, Q(296 K), n_air range) of the three gas families
GAS_FAMILIES = {
    "H2O": (1, 18.01, 174.0, (0.60, 0.80)),
    "CO2": (2, 43.99, 286.0, (0.65, 0.80)),
    "O3": (3, 47.98, 3483.0, (0.65, 0.80)),
}


def tips_power_law(q296: float, t_min: float = 70.0, t_max: float = 3000.0,
                   t_step: float = 1.0) -> Tuple[np.ndarray, np.ndarray]:
    """Partition-sum table Q(T) = Q296 (T/296)^1.5 on a regular temperature grid."""
    t = np.arange(t_min, t_max + 0.5 * t_step, t_step, dtype=np.float64)
    return t, q296 * (t / 296.0) ** 1.5


def _draw_lines(rng: np.random.Generator, n: int, nu_lo: float, nu_hi: float,
                mol_id: int, n_air_range: Tuple[float, float]) -> Dict[str, np.ndarray]:
    return {
        "nu0": rng.uniform(nu_lo, nu_hi, n),
        "Sref": 10.0 ** rng.uniform(-26.0, -19.0, n),
        "g_air": rng.uniform(0.06, 0.09, n),
        "g_self": rng.uniform(0.08, 0.12, n),
        "Elow": rng.uniform(0.0, 3000.0, n),
        "n_air": rng.uniform(n_air_range[0], n_air_range[1], n),
        "shift": rng.uniform(-0.004, 0.0, n),
        "mol_id": np.full(n, mol_id, dtype=np.int32),
        "iso_id": np.ones(n, dtype=np.int32),
    }


def co2_band(n_lines: int = 2000, nu_lo: float = 700.0, nu_hi: float = 750.0,
             seed: int = 700750) -> SpectralData:
    """CO2-like band: one isotopologue (2,1), M = 43.99, Q(296) = 286."""
    rng = np.random.default_rng(seed)
    mol, mass, q296, nrange = GAS_FAMILIES["CO2"]
    lines = _draw_lines(rng, n_lines, nu_lo, nu_hi, mol, nrange)
    return SpectralData(lines, {(mol, 1): tips_power_law(q296)}, {(mol, 1): mass}, "CO2")


def three_gas_lines(n_lines: int = 200_000, nu_lo: float = 600.0, nu_hi: float = 2500.0,
                    shares: Sequence[float] = (0.5, 0.3, 0.2), seed: int = 6002500) -> SpectralData:
    """H2O-, CO2- and O3-like lines split by ``shares``, centres uniform in [nu_lo, nu_hi]."""
    rng = np.random.default_rng(seed)
    parts: List[Dict[str, np.ndarray]] = []
    tips, masses = {}, {}
    counts = [int(round(s * n_lines)) for s in shares]
    counts[-1] = n_lines - sum(counts[:-1])
    for (name, (mol, mass, q296, nrange)), n in zip(GAS_FAMILIES.items(), counts):
        parts.append(_draw_lines(rng, n, nu_lo, nu_hi, mol, nrange))
        tips[(mol, 1)] = tips_power_law(q296)
        masses[(mol, 1)] = mass
    lines = {k: np.concatenate([p[k] for p in parts]) for k in parts[0]}
    return SpectralData(lines, tips, masses, None)


def restrict(sd: SpectralData, nu_lo: float, nu_hi: float) -> SpectralData:
    """Lines with nu0 in [nu_lo, nu_hi] (tables and masses kept)."""
    keep = (sd.lines["nu0"] >= nu_lo) & (sd.lines["nu0"] <= nu_hi)
    return SpectralData({k: v[keep].copy() for k, v in sd.lines.items()},
                        dict(sd.tips), dict(sd.molar_masses), sd.molecule)


def scale_strengths(sd: SpectralData, factor: float) -> SpectralData:
    """Same lines with Sref multiplied by ``factor`` (optically thin variants)."""
    lines = {k: v.copy() for k, v in sd.lines.items()}
    lines["Sref"] = lines["Sref"] * factor
    return SpectralData(lines, dict(sd.tips), dict(sd.molar_masses), sd.molecule)


def logp_levels(n_levels: int = 61) -> Dict[str, np.ndarray]:
    """Levels uniform in ln p between the USSA76 surface and 50 km pressures.

    Temperature and altitude are linear in ln p between the USSA76 table points;
    O3 follows the AFGL log-VMR table at those altitudes, CO2 is 415 ppm and
    H2O = 1e-2 exp(-z / 2 km). Returned TOA first (pressure increasing).
    """
    lnp_tab = np.log(USSA_P_HPA[::-1])            # increasing
    lnp = np.linspace(lnp_tab[0], lnp_tab[-1], n_levels)
    p = np.exp(lnp)
    p[0], p[-1] = USSA_P_HPA[-1], USSA_P_HPA[0]
    t = np.interp(lnp, lnp_tab, USSA_T_K[::-1])
    z = np.interp(lnp, lnp_tab, USSA_ALT_KM[::-1])
    return {
        "p": p, "t": t, "z": z,
        "H2O": 1e-2 * np.exp(-z / 2.0),
        "CO2": np.full(n_levels, 415e-6),
        "O3": log_vmr_interp(z, "O3"),
    }


def logp_profile(n_levels: int = 61) -> AtmosphericProfile:
    """60-layer (by default) profile of ``logp_levels`` with H2O, CO2 and O3."""
    lv = logp_levels(n_levels)
    return AtmosphericProfile(lv["p"], lv["t"], {g: lv[g] for g in ("H2O", "CO2", "O3")})


def ussa_levels() -> Dict[str, np.ndarray]:
    """The 21-level USSA76 profile with H2O, CO2 and O3 as arrays, TOA first."""
    prof = us_standard_atmosphere(["H2O", "CO2", "O3"])
    z = USSA_ALT_KM[::-1].copy()
    return {"p": prof.pressure_hpa, "t": prof.temperature_k, "z": z,
            **{g: prof.vmr[g] for g in ("H2O", "CO2", "O3")}}


def perturbed_levels(base: Dict[str, np.ndarray], n_profiles: int, seed: int,
                     t_sigma: float = 5.0, corr_levels: float = 3.0,
                     h2o_log_sigma: float = 0.3, t_offset: float = 0.0) -> Dict[str, np.ndarray]:
    """Batch of profiles around ``base``.

    Temperatures get Gaussian perturbations (sigma ``t_sigma`` K, Gaussian
    correlation ``corr_levels`` levels, drawn through a Cholesky factor) plus
    ``t_offset``; H2O is scaled per profile by exp(N(0, h2o_log_sigma)) and
    clipped to 1. Returns arrays shaped [n_profiles, n_levels].
    """
    rng = np.random.default_rng(seed)
    n_lev = base["p"].size
    i = np.arange(n_lev)
    cov = t_sigma ** 2 * np.exp(-0.5 * ((i[:, None] - i[None, :]) / corr_levels) ** 2)
    chol = np.linalg.cholesky(cov + 1e-9 * np.eye(n_lev))
    dt = rng.standard_normal((n_profiles, n_lev)) @ chol.T
    scale = np.exp(h2o_log_sigma * rng.standard_normal(n_profiles))
    out = {
        "p": np.broadcast_to(base["p"], (n_profiles, n_lev)).copy(),
        "t": base["t"][None, :] + dt + t_offset,
        "H2O": np.minimum(base["H2O"][None, :] * scale[:, None], 1.0),
        "CO2": np.broadcast_to(base["CO2"], (n_profiles, n_lev)).copy(),
        "O3": np.broadcast_to(base["O3"], (n_profiles, n_lev)).copy(),
    }
    return out


def profile_from_levels(levels: Dict[str, np.ndarray], i: int | None = None,
                        gases: Sequence[str] = ("H2O", "CO2", "O3")) -> AtmosphericProfile:
    """AtmosphericProfile for one row (``i``) of a batch, or for unbatched levels."""
    pick = (lambda a: a) if i is None else (lambda a: a[i])
    return AtmosphericProfile(pick(levels["p"]), pick(levels["t"]),
                              {g: pick(levels[g]) for g in gases})
