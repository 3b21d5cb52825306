"""CPU restatement of the surrogate network's training step — TEST INFRASTRUCTURE ONLY.

The surrogate has no reference counterpart (the reference, PyLBLRTM 0.1.2, has no
learned component); this module is the checker for the device network in
``pylblrtm_b200/surrogate.py`` and ``pylblrtm_b200/csrc/mlp.cu``. It states the same
arithmetic in numpy: bf16 values (round to nearest even) at exactly the points where
the device stores bf16 -- standardised inputs, weights, pre-activations z, activations
gelu(z), and output-layer / hidden-layer gradients dz -- with products accumulated in
float64 (the device accumulates in float32, so results agree to accumulation-order
rounding, not bit for bit). With ``rounding=False`` every bf16 rounding is skipped,
which is how the hand-written backward pass is checked against torch autograd.
Layer l computes z_l = x_l W_l^T + b_l; hidden layers y = gelu(z) (erf form); the
output is p = sigmoid(z) with loss sum (p - t)^2 and gradient scale s:
dz_out = s * 2 (p - t) p (1 - p).
"""

from __future__ import annotations

import math
from typing import List, Sequence, Tuple

import numpy as np

try:
    from scipy.special import erf as _erf
except ImportError:  # pragma: no cover
    _erf = np.vectorize(math.erf)


def bf16(x) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest, ties to even), returned as float32."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).reshape(a.shape)


def gelu(z):
    return 0.5 * z * (1.0 + _erf(z / math.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + _erf(z / math.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / math.sqrt(2.0 * math.pi)


def forward_backward(raw: np.ndarray, target: np.ndarray, mean: np.ndarray, inv_std: np.ndarray,
                     w: Sequence[np.ndarray], b: Sequence[np.ndarray], grad_scale: float,
                     rounding: bool = True) -> Tuple[float, np.ndarray, List[np.ndarray], List[np.ndarray]]:
    """(sum of squared errors, p, [dW_l], [db_l]) of one batch.

    ``w[l]`` is [N_l, K_l] float32 (unpadded), ``b[l]`` [N_l]; ``raw`` [B, K_0].
    """
    rnd = bf16 if rounding else (lambda v: np.asarray(v, np.float64))
    f32 = (lambda v: np.asarray(v, np.float32)) if rounding else (lambda v: np.asarray(v, np.float64))
    L = len(w)
    wb = [rnd(wl).astype(np.float64) for wl in w]
    x = [rnd(f32((f32(raw) - f32(mean)) * f32(inv_std))).astype(np.float64)]
    zs = []
    p = None
    for l in range(L):
        z = f32(x[l] @ wb[l].T) + f32(b[l])
        if l < L - 1:
            zs.append(rnd(z).astype(np.float64))
            x.append(rnd(f32(gelu(np.asarray(z, np.float64)))).astype(np.float64))
        else:
            p = 1.0 / (1.0 + np.exp(-np.asarray(z, np.float64)))
    d = p - target
    sse = float(np.sum(d * d))
    dz = rnd(f32(grad_scale * 2.0 * d * p * (1.0 - p))).astype(np.float64)
    dw: List[np.ndarray] = [None] * L
    db: List[np.ndarray] = [None] * L
    for l in range(L - 1, -1, -1):
        dw[l] = dz.T @ x[l]
        db[l] = dz.sum(0)
        if l > 0:
            dx = f32(dz @ wb[l])
            dz = rnd(f32(np.asarray(dx, np.float64) * gelu_grad(zs[l - 1]))).astype(np.float64)
    return sse, p, dw, db


def adam(w, m, v, g, step: int, lr: float, b1: float = 0.9, b2: float = 0.999, eps: float = 1e-8):
    """One bias-corrected Adam step in float32; returns (w, m, v)."""
    w, m, v, g = (np.asarray(a, np.float32) for a in (w, m, v, g))
    c1 = np.float32(1.0 / (1.0 - b1 ** step))
    c2 = np.float32(1.0 / (1.0 - b2 ** step))
    m = np.float32(b1) * m + np.float32(1.0 - b1) * g
    v = np.float32(b2) * v + np.float32(1.0 - b2) * g * g
    w = w - np.float32(lr) * (m * c1) / (np.sqrt(v * c2) + np.float32(eps))
    return w, m, v
