"""Layer Jacobians of the optical depth for retrievals (no reference counterpart).

The reference forward model (``pylblrtm/forward.py:157-317``) has no
derivatives. Here one pass of a hand-written kernel (``lbl_jacobian_ml_f32``)
gives, for every layer k and grid point, d tau / d T_k and d tau / d ln VMR_k of
one gas (the layer quantities the reference builds in
``atmosphere.py:110-141``; the column scales with the VMR). A layer's T and VMR
enter only that layer's optical depth, so these per-layer arrays are the whole
Jacobian of tau = sum_k od_k. The same kernel in vector-Jacobian mode backs
:func:`layer_optical_depth`, a ``torch.autograd.Function`` whose backward pass
recomputes the Voigt values instead of storing the Jacobian.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Dict, Optional, Sequence

import numpy as np

from . import engine
from .atmosphere import COLUMN_FACTOR, AtmosphericProfile
from .spectral_data import SpectralData


def layer_jacobians(spectral_data: SpectralData, profile: AtmosphericProfile, nu_min_cm1: float,
                    nu_max_cm1: float, *, step_cm1: float = 0.001, line_cutoff_cm1: float = 25.0,
                    tile_width_cm1: float = 2.0, gas: str = "H2O", as_numpy: bool = True,
                    deterministic: bool = False) -> Dict[str, object]:
    """Per-layer optical depth and its Jacobians for one profile.

    Returns ``nu`` [n], ``od`` [n_layers, n], ``dtau_dT`` [n_layers, n]
    (per K of the layer temperature) and ``dtau_dlnvmr`` [n_layers, n] (per unit
    of ln VMR of ``gas`` in the layer), computed in float32 engine arithmetic.
    """
    if not isinstance(spectral_data, SpectralData):
        raise TypeError("spectral_data must be a SpectralData instance")
    if not isinstance(profile, AtmosphericProfile):
        raise TypeError("profile must be an AtmosphericProfile instance")
    if gas not in profile.vmr:
        raise ValueError(f"gas '{gas}' is not in the profile")
    grid = engine.make_grid(nu_min_cm1, nu_max_cm1, step_cm1, tile_width_cm1)
    job = engine.Job(spectral_data, engine.layer_input_from_profile(profile), grid, float(line_cutoff_cm1),
                     warn_level=3)
    od, d_t, d_v = job.jacobian(gas, deterministic=deterministic)
    out = {"nu": grid.nu, "od": od[0], "dtau_dT": d_t[0], "dtau_dlnvmr": d_v[0]}
    if as_numpy:
        out = {k: (v if isinstance(v, np.ndarray) else v.double().cpu().numpy()) for k, v in out.items()}
    return out


def layer_jacobians_batch(spectral_data: SpectralData, pressure_hpa, temperature_k, vmr: Dict[str, object],
                          nu_min_cm1: float, nu_max_cm1: float, *, step_cm1: float = 0.001,
                          line_cutoff_cm1: float = 25.0, tile_width_cm1: float = 2.0, gas: str = "H2O",
                          mu_view=1.0, profiles_per_launch: int = 32, on_chunk=None,
                          deterministic: bool = False) -> Optional[Dict[str, object]]:
    """Transmittance and per-layer Jacobians of a batch of level profiles.

    ``pressure_hpa``, ``temperature_k`` and every ``vmr[gas]`` are ``[n, n_levels]``
    (TOA first, validated like ``transmittance_batch``); ``mu_view`` is a scalar or one
    value per profile. For each chunk of ``profiles_per_launch`` profiles the device
    computes ``od``, ``dtau_dT`` and ``dtau_dlnvmr`` ``[m, n_layers, n_nu]`` (float32)
    and ``trans`` ``[m, n_nu]`` = exp(-sum_k od_k / mu) (float64). With ``on_chunk``
    each chunk is handed to ``on_chunk(profile_slice, outputs)`` as device tensors and
    nothing is kept (for batches whose Jacobians exceed device memory); otherwise the
    chunks are concatenated on the device and returned with ``nu``.
    """
    import torch
    from .batch import _validate_levels
    if not isinstance(spectral_data, SpectralData):
        raise TypeError("spectral_data must be a SpectralData instance")
    p = np.atleast_2d(np.asarray(pressure_hpa, dtype=np.float64))
    t = np.atleast_2d(np.asarray(temperature_k, dtype=np.float64))
    gases = list(vmr.keys())
    v = {g: np.atleast_2d(np.asarray(vmr[g], dtype=np.float64)) for g in gases}
    _validate_levels(p, t, v)
    if gas not in v:
        raise ValueError(f"gas '{gas}' is not in vmr")
    if nu_min_cm1 >= nu_max_cm1:
        raise ValueError("nu_min_cm1 must be strictly less than nu_max_cm1")
    if step_cm1 <= 0:
        raise ValueError("step_cm1 must be positive")
    n = p.shape[0]
    mu = np.broadcast_to(np.asarray(mu_view, dtype=np.float64), (n,)).copy()
    if not np.all((mu > 0.0) & (mu <= 1.0)):
        raise ValueError("mu_view must be in (0, 1]")
    if profiles_per_launch < 1:
        raise ValueError("profiles_per_launch must be >= 1")
    grid = engine.make_grid(nu_min_cm1, nu_max_cm1, step_cm1, tile_width_cm1)
    vmr_all = np.stack([v[g] for g in gases], axis=1)
    keep = []
    for b0 in range(0, n, profiles_per_launch):
        sl = slice(b0, min(n, b0 + profiles_per_launch))
        li = engine.LayerInput(gases=gases, levels_p=p[sl], levels_t=t[sl], levels_vmr=vmr_all[sl])
        job = engine.Job(spectral_data, li, grid, float(line_cutoff_cm1), warn_level=3)
        od, d_t, d_v = job.jacobian(gas, deterministic=deterministic)
        m = od.shape[0]
        trans = torch.empty((m, grid.n_nu), dtype=torch.float64, device=od.device)
        mu_d = torch.as_tensor(mu[sl], device=od.device)
        if od.shape[1] > 0:
            from . import _lib
            _lib.call("lbl_layer_sum_exp_f32", od.data_ptr(), m, od.shape[1], grid.n_nu, mu_d.data_ptr(),
                      trans.data_ptr(), 0, torch.cuda.current_stream().cuda_stream)
        else:
            trans.fill_(1.0)
        out = {"od": od, "dtau_dT": d_t, "dtau_dlnvmr": d_v, "trans": trans}
        if on_chunk is not None:
            on_chunk(sl, out)
        else:
            keep.append(out)
    if on_chunk is not None:
        return None
    res = {k: torch.cat([c[k] for c in keep]) for k in keep[0]}
    res["nu"] = grid.nu
    return res


@dataclass
class LayerState:
    """Fixed inputs of :func:`layer_optical_depth` (everything but T and ln VMR).

    Arrays are [n_prof, n_layers]; ``vmr`` holds every gas of the profiles (the
    differentiated gas's entry is replaced by exp(ln VMR) on each call);
    ``air_col`` is the dry-air column of each layer [molec cm^-2].
    """
    spectral_data: SpectralData
    p_atm: np.ndarray
    air_col: np.ndarray
    vmr: Dict[str, np.ndarray]
    gas: str
    grid: engine.Grid
    cutoff: float = 25.0

    @classmethod
    def from_profiles(cls, spectral_data: SpectralData, profiles: Sequence[AtmosphericProfile], gas: str,
                      nu_min_cm1: float, nu_max_cm1: float, step_cm1: float = 0.001,
                      line_cutoff_cm1: float = 25.0, tile_width_cm1: float = 2.0) -> "LayerState":
        lays = [p.build_layers() for p in profiles]
        gases = list(profiles[0].vmr.keys())
        p_atm = np.stack([lay.pressure_atm for lay in lays])
        # dry-air column, formed like atmosphere.py:133-135
        air = np.stack([COLUMN_FACTOR * (np.abs(np.diff(p.pressure_hpa)) * 100.0) / 1e4 for p in profiles])
        vmr = {g: np.stack([lay.vmr[g] for lay in lays]) for g in gases}
        grid = engine.make_grid(nu_min_cm1, nu_max_cm1, step_cm1, tile_width_cm1)
        return cls(spectral_data, p_atm, air, vmr, gas, grid, float(line_cutoff_cm1))

    def layer_input(self, t_layer: np.ndarray, lnvmr: np.ndarray) -> engine.LayerInput:
        gases = list(self.vmr.keys())
        vmr = dict(self.vmr)
        vmr[self.gas] = np.exp(lnvmr)
        v = np.stack([vmr[g] for g in gases], axis=1)
        col = v * self.air_col[:, None, :]
        return engine.LayerInput(gases=gases, layer_p=self.p_atm, layer_t=t_layer, layer_vmr=v, layer_col=col)


def _torch_function():
    import torch

    class LayerOpticalDepth(torch.autograd.Function):
        """tau[b, nu] = sum_k od_k(T_k, ln VMR_k) for a batch of profiles (float64 out).

        forward(t_layer [B, L], lnvmr_layer [B, L], state) runs the multi-level
        float32 engine; backward runs the Jacobian kernel in vector-Jacobian mode
        (Voigt values recomputed, no stored Jacobian).
        """

        @staticmethod
        def forward(ctx, t_layer, lnvmr_layer, state):
            t_np = t_layer.detach().double().cpu().numpy()
            v_np = lnvmr_layer.detach().double().cpu().numpy()
            job = engine.Job(state.spectral_data, state.layer_input(t_np, v_np), state.grid, state.cutoff)
            res = job.run("fp32", want_od=False, want_tau=True)
            ctx.state = state
            ctx.save_for_backward(t_layer.detach(), lnvmr_layer.detach())
            return res.tau.to(t_layer.device)

        @staticmethod
        def backward(ctx, g):
            t_layer, lnvmr = ctx.saved_tensors
            state = ctx.state
            job = engine.Job(state.spectral_data,
                             state.layer_input(t_layer.double().cpu().numpy(), lnvmr.double().cpu().numpy()),
                             state.grid, state.cutoff)
            vt, vv = job.jacobian(state.gas, g_tau=g)
            return vt.to(t_layer.device, t_layer.dtype), vv.to(lnvmr.device, lnvmr.dtype), None

    return LayerOpticalDepth


_FN = None


def layer_optical_depth(t_layer, lnvmr_layer, state: LayerState):
    """Differentiable tau [B, n] from layer temperatures and ln VMR (torch tensors)."""
    global _FN
    if _FN is None:
        _FN = _torch_function()
    return _FN.apply(t_layer, lnvmr_layer, state)
