"""Float64 torch restatement of the forward model with autograd — TEST INFRASTRUCTURE ONLY.

Follows the same reference lines as ``oracle/restate.py`` (``pylblrtm/forward.py:
157-317``, ``spectral_data.py:43-52``) but in torch float64, so that autograd gives
d od_k / d T_k and d od_k / d ln VMR_k as an independent check of the engine's
hand-written Jacobians. The Faddeeva function is Weideman's (1994) rational
approximation (SIAM J. Numer. Anal. 31:1497-1518), N = 36, in complex128 (relative
error ~1e-14 against scipy.special.wofz over the upper half plane); its coefficients
are computed here from the published construction, independently of the engine's
table. Tile-window membership is decided on detached values, like the reference's
boolean masks.
"""

from __future__ import annotations

import math
from typing import Dict, Tuple

import numpy as np
import torch

from .restate import C2, DOPPLER, SQRT_LN2, T_REF, VOIGT_K, prepare_groups

_N = 36


def _weideman_coefficients(n: int = _N) -> Tuple[float, np.ndarray]:
    m = 2 * n
    k = np.arange(-m + 1, m)
    big_l = math.sqrt(n / math.sqrt(2.0))
    t = big_l * np.tan(k * np.pi / m / 2.0)
    f = np.concatenate([[0.0], np.exp(-t ** 2) * (big_l ** 2 + t ** 2)])
    a = np.real(np.fft.fft(np.fft.fftshift(f))) / (2 * m)
    return big_l, a[1:n + 1]


_L, _A = _weideman_coefficients()


def faddeeva(z: torch.Tensor) -> torch.Tensor:
    """w(z) for Im z >= 0 (complex128), differentiable."""
    big_l = torch.tensor(_L, dtype=torch.complex128)
    d = big_l - 1j * z
    zz = (big_l + 1j * z) / d
    p = torch.zeros_like(z) + float(_A[-1])
    for c in _A[-2::-1]:
        p = p * zz + float(c)
    return 2.0 * p / d ** 2 + (1.0 / math.sqrt(math.pi)) / d


def _interp(x: torch.Tensor, xp: np.ndarray, fp: np.ndarray) -> torch.Tensor:
    """np.interp with a gradient in x (clamped ends)."""
    xp_t = torch.tensor(xp, dtype=torch.float64)
    fp_t = torch.tensor(fp, dtype=torch.float64)
    if x.item() >= xp[-1]:
        return fp_t[-1] + 0.0 * x
    if x.item() < xp[0]:
        return fp_t[0] + 0.0 * x
    j = int(np.searchsorted(xp, x.item(), side="right") - 1)
    slope = (fp_t[j + 1] - fp_t[j]) / (xp_t[j + 1] - xp_t[j])
    return slope * (x - xp_t[j]) + fp_t[j]


def layer_optical_depth(nu: np.ndarray, lines: Dict[str, np.ndarray], tips, masses, p_atm: np.ndarray,
                        t_layer: torch.Tensor, vmr_layer: Dict[str, torch.Tensor], air_col: np.ndarray,
                        k: int, cutoff: float = 25.0, tile_width: float = 2.0) -> torch.Tensor:
    """od_k(nu) [n] of layer k; t_layer [n_layers] and vmr_layer[gas] [n_layers] are tensors.

    The column of each gas is vmr_layer[gas] * air_col (atmosphere.py:137-139).
    """
    n_nu = nu.size
    step = float(nu[1] - nu[0]) if n_nu > 1 else 0.001
    tile = max(1, int(np.floor(tile_width / step + 1e-8)))
    t_np = t_layer.detach().numpy()
    prepared = prepare_groups(nu, lines, tips, masses, tuple(vmr_layer.keys()), p_atm, t_np, cutoff)
    nu_t = torch.tensor(nu, dtype=torch.float64)
    od = torch.zeros(n_nu, dtype=torch.float64)
    T = t_layer[k]
    P = float(p_atm[k])
    for mol_id, iso_id, gas, mask, mm, _ in prepared:
        vmr = vmr_layer[gas][k]
        col = vmr * float(air_col[k])
        if col.item() == 0.0:
            continue
        t_arr, q_arr = tips[(int(mol_id), int(iso_id))]
        q_ratio = _interp(torch.tensor(T_REF, dtype=torch.float64), t_arr, q_arr) / _interp(T, t_arr, q_arr)
        p_self = vmr * P
        p_air = P - p_self
        idx = np.flatnonzero(mask)
        c = torch.tensor(lines["nu0"][idx])
        shifted = c + torch.tensor(lines["shift"][idx]) * p_air
        r_c = shifted * torch.tanh(0.5 * C2 * shifted / T)
        strength = (torch.tensor(lines["Sref"][idx]) * q_ratio
                    * torch.exp(-C2 * torch.tensor(lines["Elow"][idx]) * (1.0 / T - 1.0 / T_REF))
                    * (-torch.expm1(-C2 * c / T)) / (-torch.expm1(-C2 * c / T_REF)) * col / r_c)
        lorentz = (T_REF / T) ** torch.tensor(lines["n_air"][idx]) * (
            torch.tensor(lines["g_air"][idx]) * p_air + torch.tensor(lines["g_self"][idx]) * p_self)
        doppler = c * DOPPLER * torch.sqrt(T / mm)
        sh_np = shifted.detach().numpy()
        for t0 in range(0, n_nu, tile):
            t1 = min(t0 + tile, n_nu)
            near = (sh_np >= nu[t0] - cutoff) & (sh_np <= nu[t1 - 1] + cutoff)
            if not near.any():
                continue
            b = np.flatnonzero(near)
            z = SQRT_LN2 * ((nu_t[t0:t1, None] - shifted[b]) + 1j * lorentz[b]) / doppler[b]
            phi = faddeeva(z).real * (VOIGT_K / doppler[b])
            od = od + torch.cat([torch.zeros(t0, dtype=torch.float64), phi @ strength[b],
                                 torch.zeros(n_nu - t1, dtype=torch.float64)])
    return od * nu_t * torch.tanh(0.5 * C2 * nu_t / T)
