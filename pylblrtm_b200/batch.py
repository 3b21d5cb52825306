"""Batched forward model: many atmospheric profiles against one line list.

``transmittance_batch`` evaluates a batch of level profiles (same levels count
and gases) in one pass of the device pipeline: the per-layer records and the
summation kernels take ``n_profiles * n_layers`` rows, so a batch costs one
launch per stage. Results for each profile equal ``compute_transmittance`` on
that profile alone, with one documented difference: the reference's band mask
(``pylblrtm/forward.py:190-220``) uses the largest layer pressure of the whole
batch, which can only add lines that no tile window admits (so the spectra are
unchanged) but can add a molar-mass warning for a group that a single profile
would not reach.

With ``channel_width_cm1`` the transmittance is box-averaged on the device into
consecutive half-open channels of ``round(channel_width / step)`` grid points
starting at ``nu_min`` (an incomplete last channel is dropped), without storing
the per-point spectrum.
"""

from __future__ import annotations

from typing import Dict, Optional, Tuple

import numpy as np

from . import engine
from .spectral_data import SpectralData

MAX_ROWS_PER_LAUNCH = 65535     # grid y-dimension of the summation kernels


def _validate_levels(p: np.ndarray, t: np.ndarray, vmr: Dict[str, np.ndarray]) -> None:
    """Vectorised form of AtmosphericProfile's checks (pylblrtm/atmosphere.py:72-95)."""
    if p.ndim != 2 or p.shape[1] < 2:
        raise ValueError("pressure_hpa must be [n_profiles, n_levels] with at least 2 levels")
    if not np.all(np.isfinite(p)) or np.any(p <= 0):
        raise ValueError("pressure_hpa must be finite and positive")
    if np.any(np.diff(p, axis=1) <= 0):
        raise ValueError("pressure_hpa must be strictly increasing from TOA "
                         "(smallest pressure = highest altitude = index 0)")
    if t.shape != p.shape:
        raise ValueError("temperature_k must have the same shape as pressure_hpa")
    if not np.all(np.isfinite(t)) or np.any(t <= 0):
        raise ValueError("temperature_k must be finite and positive")
    for gas, v in vmr.items():
        if v.shape != p.shape:
            raise ValueError(f"vmr['{gas}'] must have the same shape as pressure_hpa {p.shape}, got {v.shape}")
        if not np.all(np.isfinite(v)) or np.any(v < 0) or np.any(v > 1):
            raise ValueError(f"vmr['{gas}'] must be finite and in [0, 1]")


def transmittance_batch(
    spectral_data: SpectralData,
    pressure_hpa,
    temperature_k,
    vmr: Dict[str, object],
    nu_min_cm1: float,
    nu_max_cm1: float,
    *,
    step_cm1: float = 0.001,
    line_cutoff_cm1: float = 25.0,
    tile_width_cm1: float = 2.0,
    mu_view=1.0,
    precision: str = "fp32",
    channel_width_cm1: Optional[float] = None,
    profiles_per_launch: Optional[int] = None,
    as_numpy: bool = True,
    deterministic: bool = False,
) -> Tuple[np.ndarray, object]:
    """Transmittance of a batch of profiles.

    ``pressure_hpa``, ``temperature_k`` and every ``vmr[gas]`` are
    ``[n_profiles, n_levels]`` (TOA first); ``mu_view`` is a scalar or one value
    per profile. Returns ``(nu, T[n_profiles, n_nu])`` or, with
    ``channel_width_cm1``, ``(channel_centres, T[n_profiles, n_channels])``.
    ``as_numpy=False`` keeps the result on the device (a torch tensor);
    ``deterministic`` as in ``compute_transmittance``.
    """
    if not isinstance(spectral_data, SpectralData):
        raise TypeError("spectral_data must be a SpectralData instance")
    p = np.atleast_2d(np.asarray(pressure_hpa, dtype=np.float64))
    t = np.atleast_2d(np.asarray(temperature_k, dtype=np.float64))
    gases = list(vmr.keys())
    v = {g: np.atleast_2d(np.asarray(vmr[g], dtype=np.float64)) for g in gases}
    _validate_levels(p, t, v)
    if nu_min_cm1 >= nu_max_cm1:
        raise ValueError("nu_min_cm1 must be strictly less than nu_max_cm1")
    if step_cm1 <= 0:
        raise ValueError("step_cm1 must be positive")
    n_prof, n_lev = p.shape
    mu = np.broadcast_to(np.asarray(mu_view, dtype=np.float64), (n_prof,)).copy()
    if not np.all((mu > 0.0) & (mu <= 1.0)):
        raise ValueError("mu_view must be in (0, 1]")
    grid = engine.make_grid(nu_min_cm1, nu_max_cm1, step_cm1, tile_width_cm1)
    channels = None
    if channel_width_cm1 is not None:
        width = int(round(channel_width_cm1 / step_cm1))
        if width < 1 or grid.n_nu // width < 1:
            raise ValueError("channel_width_cm1 must cover at least one grid point and fit the grid")
        channels = (width, grid.n_nu // width)
    n_lay = n_lev - 1
    limit = max(1, MAX_ROWS_PER_LAUNCH // max(n_lay, 1))
    chunk = min(profiles_per_launch or limit, limit)
    vmr_all = np.stack([v[g] for g in gases], axis=1) if gases else np.zeros((n_prof, 0, n_lev))
    outs = []
    import torch
    for b0 in range(0, n_prof, chunk):
        b1 = min(b0 + chunk, n_prof)
        li = engine.LayerInput(gases=gases, levels_p=p[b0:b1], levels_t=t[b0:b1], levels_vmr=vmr_all[b0:b1])
        job = engine.Job(spectral_data, li, grid, float(line_cutoff_cm1), warn_level=3)
        res = job.run(precision, mu=mu[b0:b1], want_od=False, want_trans=channels is None, channels=channels,
                      deterministic=deterministic)
        outs.append(res.channels if channels is not None else res.trans)
    if not outs:                    # no profiles (e.g. a rank's empty share): an empty result
        n_out = channels[1] if channels is not None else grid.n_nu
        out = engine._torch().empty((0, n_out), dtype=torch.float64, device="cuda")
    else:
        out = torch.cat(outs, dim=0) if len(outs) > 1 else outs[0]
    if channels is not None:
        width, n_ch = channels
        axis = grid.nu_min + (np.arange(n_ch) * width + 0.5 * (width - 1)) * grid.step
    else:
        axis = grid.nu
    return axis, (engine.to_host(out) if as_numpy else out)
