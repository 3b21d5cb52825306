"""Channel-transmittance surrogate trained on the engine's own spectra (no reference counterpart).

A multilayer perceptron maps one 20-layer profile (20 layer temperatures, 20 ln VMR
of H2O, 20 ln VMR of CO2, and the view cosine mu: 61 standardised inputs) to the
channel-mean transmittance of 2,000 channels of 0.25 cm^-1 over 650-1150 cm^-1.
Training targets come from the line-by-line engine (``engine.Job.run`` with channel
box-averaging), so the network learns this library's own forward model.

Everything numeric runs in ``liblblgpu.so`` (include/lblgpu.h):
  * ``lbl_gemm_bf16`` -- BF16 tensor-core GEMM (tcgen05, TMA, float32 accumulators in
    tensor memory) with fused epilogues: bias + GELU (forward), bias + sigmoid + MSE
    gradient (output layer), GELU' (backward), float32 split-K partials (weight grads);
  * ``lbl_adam_step`` -- Adam on float32 master weights that refreshes the bf16
    weights and their transposes; ``lbl_rowsum_bf16`` -- bias gradients;
  * ``lbl_pack_inputs_bf16`` -- standardisation; ``lbl_ensemble_gate`` -- ensemble
    mean, spread and gate flag.
Every GEMM is "A . B^T" with both operands K-contiguous, so the backward pass keeps
transposed copies: W and W^T, activations X and X^T, output gradients dZ and dZ^T.
Widths are padded to multiples of 128 (inputs 61 -> 128, outputs 2000 -> 2048); the
padding stays zero through training (its gradients are zero).

:class:`GatedSurrogate` evaluates a 4-member ensemble; a profile whose ensemble spread
(max over channels of the members' standard deviation, times a calibration factor)
exceeds the gate is recomputed by the float32 line-by-line engine.
"""

from __future__ import annotations

import ctypes
import math
import time
from dataclasses import dataclass
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import _lib, engine, synthetic
from .spectral_data import SpectralData

PAD = 128
GASES = ("H2O", "CO2", "O3")


def _pad(n: int, m: int = PAD) -> int:
    return (n + m - 1) // m * m


# ---------------------------------------------------------------------------
# Profiles, features and engine-generated targets

@dataclass
class SurrogateProblem:
    """The spectral setup the surrogate replaces: grid, channels and cutoff."""
    nu_min: float = 650.0
    nu_max: float = 1150.0
    step: float = 0.001
    channel_width: float = 0.25
    cutoff: float = 25.0
    tile_width: float = 2.0

    @property
    def grid(self) -> engine.Grid:
        return engine.make_grid(self.nu_min, self.nu_max, self.step, self.tile_width)

    @property
    def channels(self) -> Tuple[int, int]:
        width = int(round(self.channel_width / self.step))
        return width, self.grid.n_nu // width

    @property
    def n_channels(self) -> int:
        return self.channels[1]


@dataclass
class ProfileBatch:
    """Layer profiles: p_atm, t [n, L]; vmr [n, 3, L] (H2O, CO2, O3); air_col [n, L]; mu [n]."""
    p_atm: np.ndarray
    t: np.ndarray
    vmr: np.ndarray
    air_col: np.ndarray
    mu: np.ndarray

    def __len__(self) -> int:
        return self.t.shape[0]

    def subset(self, idx) -> "ProfileBatch":
        return ProfileBatch(self.p_atm[idx], self.t[idx], self.vmr[idx], self.air_col[idx], self.mu[idx])

    def layer_input(self) -> engine.LayerInput:
        col = self.vmr * self.air_col[:, None, :]
        return engine.LayerInput(gases=list(GASES), layer_p=self.p_atm, layer_t=self.t, layer_vmr=self.vmr,
                                 layer_col=col)

    def features(self) -> np.ndarray:
        """[n, 61] float32: layer T, ln VMR(H2O), ln VMR(CO2), mu."""
        return np.concatenate([self.t, np.log(self.vmr[:, 0]), np.log(self.vmr[:, 1]), self.mu[:, None]],
                              axis=1).astype(np.float32)


def sample_profiles(n: int, seed: int, t_offset: float = 0.0, t_sigma: float = 5.0, corr_layers: float = 3.0,
                    h2o_log_sigma: float = 0.3, co2_log_sigma: float = 0.1,
                    mu_range: Tuple[float, float] = (0.5, 1.0)) -> ProfileBatch:
    """Perturbed 20-layer USSA76 profiles.

    Layer temperatures get correlated Gaussian perturbations (sigma ``t_sigma`` K,
    Gaussian correlation over ``corr_layers`` layers) plus ``t_offset`` (the
    out-of-distribution shift); H2O and CO2 are scaled per profile by log-normal
    factors (H2O clipped to a VMR of 1); O3 keeps the base profile; mu is uniform in
    ``mu_range``. Layers are those of the base levels (``atmosphere.py:110-141``).
    """
    lv = synthetic.ussa_levels()
    base = synthetic.profile_from_levels(lv).build_layers()
    L = base.n_layers
    rng = np.random.default_rng(seed)
    i = np.arange(L)
    cov = t_sigma ** 2 * np.exp(-0.5 * ((i[:, None] - i[None, :]) / corr_layers) ** 2)
    chol = np.linalg.cholesky(cov + 1e-9 * np.eye(L))
    t = base.temperature_k[None, :] + rng.standard_normal((n, L)) @ chol.T + t_offset
    s_h2o = np.exp(h2o_log_sigma * rng.standard_normal(n))
    s_co2 = np.exp(co2_log_sigma * rng.standard_normal(n))
    vmr = np.empty((n, 3, L))
    vmr[:, 0] = np.minimum(base.vmr["H2O"][None, :] * s_h2o[:, None], 1.0)
    vmr[:, 1] = base.vmr["CO2"][None, :] * s_co2[:, None]
    vmr[:, 2] = base.vmr["O3"][None, :]
    air = base.column_cm2["CO2"] / base.vmr["CO2"]
    mu = rng.uniform(mu_range[0], mu_range[1], n)
    return ProfileBatch(np.broadcast_to(base.pressure_atm, (n, L)).copy(), t, vmr,
                        np.broadcast_to(air, (n, L)).copy(), mu)


def engine_channels(sd: SpectralData, profiles: ProfileBatch, problem: SurrogateProblem,
                    profiles_per_launch: int = 128, as_numpy: bool = True, deterministic: bool = False):
    """Channel-mean transmittance [n, n_channels] of each profile from the float32 engine
    (``deterministic``: bit-reproducible sums, see ``compute_transmittance``)."""
    torch = engine._torch()
    grid = problem.grid
    outs = []
    for b0 in range(0, len(profiles), profiles_per_launch):
        part = profiles.subset(slice(b0, b0 + profiles_per_launch))
        job = engine.Job(sd, part.layer_input(), grid, problem.cutoff, warn_level=3)
        res = job.run("fp32", mu=part.mu, want_od=False, channels=problem.channels, deterministic=deterministic)
        outs.append(res.channels.float())
    out = torch.cat(outs) if len(outs) > 1 else outs[0]
    return out.cpu().numpy() if as_numpy else out


# ---------------------------------------------------------------------------
# Device network

class _Map:
    """TMA descriptor (host bytes) of a 2-D bf16 device tensor, which it keeps alive."""
    __slots__ = ("buf", "t", "addr")

    def __init__(self, t):
        self.t = t
        self.buf = ctypes.create_string_buffer(int(_lib.load().lbl_tensor_map_bytes()))
        self.addr = ctypes.addressof(self.buf)
        _lib.call("lbl_tensor_map_bf16", self.addr, t.data_ptr(), t.shape[0], t.shape[1], t.stride(0))


def _split_for(m: int, n: int, k: int, target_units: int = 148) -> int:
    """Split-K factor for a float32 GEMM: at least one tile per SM of the persistent
    kernel (tiles are 128 x 256, or 128 x 128 when n is not a multiple of 256), keeping
    >= 8 k-tiles of 64 per split."""
    k_tiles = k // 64
    tiles = (m // 128) * (n // (256 if n % 256 == 0 else 128))
    s = 1
    while tiles * s < target_units and k_tiles % (2 * s) == 0 and k_tiles // (2 * s) >= 8:
        s *= 2
    return s


class _Workspace:
    """Activations, gradients and their TMA maps for one batch size."""

    def __init__(self, net: "MLP", batch: int, train: bool):
        torch, dev = net.torch, net.dev
        bf = torch.bfloat16
        self.batch = batch
        dims = net.dims
        self.raw = torch.zeros((batch, net.n_in), dtype=torch.float32, device=dev)
        self.x = [torch.zeros((batch, k), dtype=bf, device=dev) for k, _ in dims]
        self.map_x = [_Map(t) for t in self.x]
        self.train = train
        if train:
            self.xt = [torch.zeros((k, batch), dtype=bf, device=dev) for k, _ in dims]
            self.z = [torch.zeros((batch, n), dtype=bf, device=dev) for _, n in dims[:-1]]
            self.dz = [torch.zeros((batch, n), dtype=bf, device=dev) for _, n in dims]
            self.dzt = [torch.zeros((n, batch), dtype=bf, device=dev) for _, n in dims]
            self.map_xt = [_Map(t) for t in self.xt]
            self.map_dz = [_Map(t) for t in self.dz]
            self.map_dzt = [_Map(t) for t in self.dzt]
            self.split = [_split_for(n, k, batch) for k, n in dims]
            self.dw = [torch.zeros((s, n, k), dtype=torch.float32, device=dev) for s, (k, n) in zip(self.split, dims)]
            self.db = [torch.zeros((n,), dtype=torch.float32, device=dev) for _, n in dims]
            self.target = torch.zeros((batch, net.n_out), dtype=torch.float32, device=dev)
            self.loss = torch.zeros((1,), dtype=torch.float64, device=dev)
        self.out = torch.zeros((batch, dims[-1][1]), dtype=torch.float32, device=dev)
        self.err = torch.zeros((1,), dtype=torch.int32, device=dev)


class MLP:
    """n_in -> hidden x depth (GELU) -> n_out (sigmoid) in BF16 with float32 accumulation.

    Weights: float32 master copies with Adam moments, bf16 copies W [N, K] and
    W^T [K, N] refreshed by every optimiser step. ``launches`` counts the kernels
    enqueued by the last call.
    """

    def __init__(self, n_in: int = 61, n_out: int = 2000, hidden: int = 1024, depth: int = 4, seed: int = 0,
                 lr: float = 1e-3, betas: Tuple[float, float] = (0.9, 0.999), eps: float = 1e-8):
        _lib.load()
        torch = engine._torch()
        self.torch = torch
        self.dev = torch.device("cuda", torch.cuda.current_device())
        if hidden % PAD:
            raise ValueError("hidden width must be a multiple of 128")
        if depth < 1:
            raise ValueError("depth must be >= 1")
        self.n_in, self.n_out, self.hidden, self.depth = int(n_in), int(n_out), int(hidden), int(depth)
        self.dims = [(_pad(n_in), hidden)] + [(hidden, hidden)] * (depth - 1) + [(hidden, _pad(n_out))]
        self.real = [(n_in, hidden)] + [(hidden, hidden)] * (depth - 1) + [(hidden, n_out)]
        self.lr, self.betas, self.eps = float(lr), tuple(float(b) for b in betas), float(eps)
        self.step = 0
        self.launches = 0
        g = torch.Generator().manual_seed(int(seed))
        w32, b32 = [], []
        for li, ((k, n), (kr, nr)) in enumerate(zip(self.dims, self.real)):
            w = torch.zeros((n, k), dtype=torch.float32)
            std = math.sqrt(2.0 / kr) if li < depth else 0.1 * math.sqrt(1.0 / kr)
            w[:nr, :kr] = torch.randn((nr, kr), generator=g) * std
            w32.append(w.to(self.dev))
            b32.append(torch.zeros((n,), dtype=torch.float32, device=self.dev))
        self.w, self.b = w32, b32
        z = lambda t: torch.zeros_like(t)
        self.mw, self.vw = [z(t) for t in w32], [z(t) for t in w32]
        self.mb, self.vb = [z(t) for t in b32], [z(t) for t in b32]
        self.w_bf = [torch.zeros((n, k), dtype=torch.bfloat16, device=self.dev) for k, n in self.dims]
        self.wt_bf = [torch.zeros((k, n), dtype=torch.bfloat16, device=self.dev) for k, n in self.dims]
        self.map_w = [_Map(t) for t in self.w_bf]
        self.map_wt = [_Map(t) for t in self.wt_bf]
        self.mean = torch.zeros((self.n_in,), dtype=torch.float32, device=self.dev)
        self.inv_std = torch.ones((self.n_in,), dtype=torch.float32, device=self.dev)
        self._ws: Dict[Tuple[int, bool], _Workspace] = {}
        self.group = None                 # data-parallel process group (None: one process)
        self.world = 1
        self.refresh_bf16()

    def data_parallel(self, group=None) -> "MLP":
        """Train data-parallel over the ranks of ``group``: rank 0's parameters and
        normalisation are broadcast, each rank's loss is scaled by 1 / (batch x world)
        and gradients are summed (all-reduce) before every Adam step."""
        from . import shard
        self.group = group
        self.world, _ = shard.world_and_rank(group)
        if self.world > 1:
            import torch.distributed as dist
            for t in self.w + self.b + [self.mean, self.inv_std]:
                dist.broadcast(t, src=dist.get_global_rank(group, 0) if group is not None else 0, group=group)
            self.refresh_bf16()
        return self

    # -- state -------------------------------------------------------------
    def refresh_bf16(self) -> None:
        """bf16 weight copies from the float32 masters (round to nearest even)."""
        for li in range(len(self.dims)):
            self.w_bf[li].copy_(self.w[li].to(self.torch.bfloat16))
            self.wt_bf[li].copy_(self.w[li].t().to(self.torch.bfloat16))

    def set_normalisation(self, mean, std) -> None:
        """Input standardisation x' = (x - mean) / std (std <= 1e-12 leaves the input at 0)."""
        mean = np.asarray(mean, np.float64)
        std = np.asarray(std, np.float64)
        inv = np.where(std > 1e-12, 1.0 / np.maximum(std, 1e-300), 0.0)
        self.mean.copy_(self.torch.as_tensor(mean, dtype=self.torch.float32))
        self.inv_std.copy_(self.torch.as_tensor(inv, dtype=self.torch.float32))

    def set_output_bias(self, p0) -> None:
        """Output bias = logit(p0) (per channel), a good start for a sigmoid output."""
        p = np.clip(np.asarray(p0, np.float64), 1e-4, 1 - 1e-4)
        b = np.zeros(self.dims[-1][1])
        b[: self.n_out] = np.log(p / (1 - p))
        self.b[-1].copy_(self.torch.as_tensor(b, dtype=self.torch.float32))

    def state_dict(self) -> dict:
        cpu = lambda ts: [t.detach().cpu().clone() for t in ts]
        return {"dims": (self.n_in, self.n_out, self.hidden, self.depth), "step": self.step,
                "lr": self.lr, "betas": self.betas, "eps": self.eps,
                "w": cpu(self.w), "b": cpu(self.b), "mw": cpu(self.mw), "vw": cpu(self.vw),
                "mb": cpu(self.mb), "vb": cpu(self.vb),
                "mean": self.mean.cpu().clone(), "inv_std": self.inv_std.cpu().clone()}

    def load_state_dict(self, st: dict) -> None:
        if tuple(st["dims"]) != (self.n_in, self.n_out, self.hidden, self.depth):
            raise ValueError(f"state has dims {st['dims']}, network has "
                             f"{(self.n_in, self.n_out, self.hidden, self.depth)}")
        for name in ("w", "b", "mw", "vw", "mb", "vb"):
            for dst, src in zip(getattr(self, name), st[name]):
                dst.copy_(src.to(self.dev))
        self.mean.copy_(st["mean"].to(self.dev))
        self.inv_std.copy_(st["inv_std"].to(self.dev))
        self.step = int(st["step"])
        self.lr, self.betas, self.eps = float(st["lr"]), tuple(st["betas"]), float(st["eps"])
        self.refresh_bf16()

    # -- device passes -----------------------------------------------------
    def workspace(self, batch: int, train: bool) -> _Workspace:
        if batch % PAD:
            raise ValueError("batch must be a multiple of 128")
        key = (batch, train)
        if key not in self._ws:
            self._ws[key] = _Workspace(self, batch, train)
        return self._ws[key]

    def _gemm(self, map_a, map_b, m, n, k, ep, ws, stream, n_split=1):
        _lib.call("lbl_gemm_bf16", map_a.addr, map_b.addr, m, n, k, n_split, ctypes.addressof(ep),
                  ws.err.data_ptr(), stream)
        self.launches += 1

    def _forward(self, ws: _Workspace, stream, train: bool, out=None) -> None:
        """Forward pass; inference writes the sigmoid output to ``out`` (float32
        [B, n_out padded], row stride n_out padded) or to the workspace."""
        B = ws.batch
        L = len(self.dims)
        _lib.call("lbl_pack_inputs_bf16", ws.raw.data_ptr(), B, self.n_in, self.mean.data_ptr(),
                  self.inv_std.data_ptr(), ws.x[0].data_ptr(), self.dims[0][0],
                  ws.xt[0].data_ptr() if train else 0, B, stream)
        self.launches += 1
        for li, (k, n) in enumerate(self.dims):
            ep = _lib.GemmEpilogue()
            ep.bias = self.b[li].data_ptr()
            if li < L - 1:
                ep.mode = _lib.GEMM_BIAS_GELU
                ep.y, ep.ld_y = ws.x[li + 1].data_ptr(), n
                if train:
                    ep.z_out, ep.ld_z = ws.z[li].data_ptr(), n
                    ep.y_t, ep.ld_yt = ws.xt[li + 1].data_ptr(), B
            else:
                ep.mode = _lib.GEMM_BIAS_SIGMOID
                ep.n_valid = self.n_out
                if train:
                    ep.target, ep.ld_target = ws.target.data_ptr(), self.n_out
                    ep.grad_scale = 1.0 / (B * self.world)
                    ep.y, ep.ld_y = ws.dz[li].data_ptr(), n
                    ep.y_t, ep.ld_yt = ws.dzt[li].data_ptr(), B
                    ep.loss = ws.loss.data_ptr()
                else:
                    ep.out_f32, ep.ld_f32 = (ws.out if out is None else out).data_ptr(), n
            self._gemm(ws.map_x[li], self.map_w[li], B, n, k, ep, ws, stream)

    def _backward(self, ws: _Workspace, stream) -> None:
        B = ws.batch
        for li in range(len(self.dims) - 1, -1, -1):
            k, n = self.dims[li]
            s = ws.split[li]
            ep = _lib.GemmEpilogue()
            ep.mode = _lib.GEMM_F32
            ep.out_f32, ep.ld_f32, ep.split_stride = ws.dw[li].data_ptr(), k, n * k
            self._gemm(ws.map_dzt[li], ws.map_xt[li], n, k, B, ep, ws, stream, n_split=s)
            _lib.call("lbl_rowsum_bf16", ws.dzt[li].data_ptr(), n, B, B, ws.db[li].data_ptr(), stream)
            self.launches += 1
            if li > 0:
                ep = _lib.GemmEpilogue()
                ep.mode = _lib.GEMM_DGELU
                ep.z_in, ep.ld_zin = ws.z[li - 1].data_ptr(), k
                ep.y, ep.ld_y = ws.dz[li - 1].data_ptr(), k
                ep.y_t, ep.ld_yt = ws.dzt[li - 1].data_ptr(), B
                self._gemm(ws.map_dz[li], self.map_wt[li], B, k, n, ep, ws, stream)

    def _adam(self, ws: _Workspace, stream, lr: float) -> None:
        self.step += 1
        b1, b2 = self.betas
        for li, (k, n) in enumerate(self.dims):
            _lib.call("lbl_adam_step", self.w[li].data_ptr(), self.mw[li].data_ptr(), self.vw[li].data_ptr(),
                      ws.dw[li].data_ptr(), ws.split[li], n * k, n, k, k, lr, b1, b2, self.eps, self.step,
                      self.w_bf[li].data_ptr(), self.wt_bf[li].data_ptr(), n, stream)
            _lib.call("lbl_adam_step", self.b[li].data_ptr(), self.mb[li].data_ptr(), self.vb[li].data_ptr(),
                      ws.db[li].data_ptr(), 1, 0, 1, n, n, lr, b1, b2, self.eps, self.step, 0, 0, 0, stream)
            self.launches += 2

    def _check(self, ws: _Workspace) -> None:
        if int(ws.err.item()) != 0:
            raise RuntimeError("lbl_gemm_bf16: a tensor-core pipeline wait timed out")

    def train_step(self, raw, target, lr: Optional[float] = None, check: bool = False):
        """One Adam step on a batch (device tensors raw [B, n_in], target [B, n_out] float32).

        Returns the device scalar of this rank's batch mean squared error (before the
        update). Data-parallel (:meth:`data_parallel`): B is the local batch.
        """
        torch = self.torch
        B = raw.shape[0]
        ws = self.workspace(B, True)
        stream = torch.cuda.current_stream().cuda_stream
        self.launches = 0
        ws.raw.copy_(raw)
        ws.target.copy_(target)
        ws.loss.zero_()
        self._forward(ws, stream, True)
        self._backward(ws, stream)
        if self.world > 1:
            from . import shard
            shard.allreduce_gradients(ws.dw + ws.db, self.group)
        self._adam(ws, stream, self.lr if lr is None else float(lr))
        if check:
            self._check(ws)
        return ws.loss / (B * self.n_out)

    def gradients(self, raw, target):
        """Forward + backward without the update: (loss, [dW], [db], output p) for tests."""
        torch = self.torch
        B = raw.shape[0]
        ws = self.workspace(B, True)
        stream = torch.cuda.current_stream().cuda_stream
        ws.raw.copy_(raw)
        ws.target.copy_(target)
        ws.loss.zero_()
        self._forward(ws, stream, True)
        self._backward(ws, stream)
        self._check(ws)
        dw = [d.sum(0)[:nr, :kr].clone() for d, (kr, nr) in zip(ws.dw, self.real)]
        db = [d[:nr].clone() for d, (_, nr) in zip(ws.db, self.real)]
        return float(ws.loss.item()) / (B * self.n_out), dw, db

    def predict(self, raw, out=None):
        """Network output [B, n_out] float32 for device inputs raw [B, n_in] (B padded to 128 inside)."""
        torch = self.torch
        B = raw.shape[0]
        Bp = _pad(B)
        ws = self.workspace(Bp, False)
        stream = torch.cuda.current_stream().cuda_stream
        self.launches = 0
        ws.raw[:B].copy_(raw)
        self._forward(ws, stream, False)
        res = ws.out[:B, : self.n_out]
        if out is not None:
            out.copy_(res)
            return out
        return res.clone()


# ---------------------------------------------------------------------------
# Ensemble, gate and fallback

def gate_threshold(est: np.ndarray, err: np.ndarray, target: float = 1e-3, quantile: float = 0.999,
                   margin: float = 0.5) -> float:
    """Largest gate t on the error estimate such that the profiles it accepts
    (est <= t) keep their ``quantile`` of the true error at or below ``target``, with
    room to spare: among the accepted, at most ``margin * (1 - quantile)`` of them may
    exceed ``target``. ``est`` and ``err`` are per-profile arrays of a calibration
    split (estimate and true max-channel error). Returns 0 when nothing qualifies."""
    est = np.asarray(est, dtype=np.float64)
    err = np.asarray(err, dtype=np.float64)
    order = np.argsort(est, kind="stable")
    e_sorted, bad = est[order], np.cumsum(err[order] > target)
    k = np.arange(1, est.size + 1)
    ok = bad <= margin * (1.0 - quantile) * k
    # a threshold must accept every profile with the same estimate: stop where est changes
    last_of_value = np.r_[e_sorted[1:] != e_sorted[:-1], True]
    cand = np.flatnonzero(ok & last_of_value)
    return float(e_sorted[cand[-1]]) if cand.size else 0.0


def channel_weights(spread: np.ndarray, err: np.ndarray, q: float = 0.99, floor: float = 1e-12) -> np.ndarray:
    """Per-channel factors that put each channel's ensemble spread on the scale of its
    true error: the ratio of their ``q`` quantiles over a calibration split
    ([n_profiles, n_channels] each), normalised to a median of 1."""
    s = np.quantile(np.asarray(spread, dtype=np.float64), q, axis=0)
    e = np.quantile(np.asarray(err, dtype=np.float64), q, axis=0)
    w = e / np.maximum(s, floor)
    w = np.where(np.isfinite(w) & (w > 0), w, 1.0)
    return (w / np.median(w)).astype(np.float32)


class GatedSurrogate:
    """4-member ensemble with a spread gate and float32-engine fallback.

    A profile is flagged when ``scale * max_c(ch_scale[c] * std_c) > gate``, std_c the
    members' spread in channel c; :func:`calibrate_gate` fits ``ch_scale`` and ``gate``
    on a calibration split so that accepted profiles meet an error target."""

    def __init__(self, members: Sequence[MLP], gate: float = 1e-3, scale: float = 1.0,
                 deterministic: bool = False, ch_scale: Optional[np.ndarray] = None):
        if not members:
            raise ValueError("at least one member")
        self.members = list(members)
        self.gate, self.scale = float(gate), float(scale)
        self.deterministic = bool(deterministic)      # of the engine fallback
        self.torch = members[0].torch
        self.launches = 0
        self.ch_scale = None
        if ch_scale is not None:
            w = np.ascontiguousarray(ch_scale, dtype=np.float32).reshape(-1)
            if w.size != members[0].n_out:
                raise ValueError(f"ch_scale needs {members[0].n_out} values, got {w.size}")
            self.ch_scale = self.torch.as_tensor(w, device=members[0].dev)

    def predictions(self, raw):
        """Every member's channel predictions [n_members, B, n_out] (device)."""
        pred, B = self._members(raw)
        return pred[:, :B, :self.members[0].n_out]

    def _members(self, raw):
        torch = self.torch
        net0 = self.members[0]
        B = raw.shape[0]
        Bp = _pad(B)
        n_pad = net0.dims[-1][1]
        pred = torch.empty((len(self.members), Bp, n_pad), dtype=torch.float32, device=net0.dev)
        self.launches = 0
        for m, net in enumerate(self.members):
            ws = net.workspace(Bp, False)
            stream = torch.cuda.current_stream().cuda_stream
            net.launches = 0
            ws.raw[:B].copy_(raw)
            if Bp > B:
                ws.raw[B:].zero_()
            net._forward(ws, stream, False, out=pred[m])
            self.launches += net.launches
        return pred, B

    def ensemble(self, raw):
        """(mean [B, n_out], est [B], flag [B] bool) on the device."""
        torch = self.torch
        net0 = self.members[0]
        pred, B = self._members(raw)
        Bp, n_pad = pred.shape[1], pred.shape[2]
        mean = torch.empty((B, net0.n_out), dtype=torch.float32, device=net0.dev)
        est = torch.empty((B,), dtype=torch.float32, device=net0.dev)
        flag = torch.empty((B,), dtype=torch.int32, device=net0.dev)
        _lib.call("lbl_ensemble_gate", pred.data_ptr(), len(self.members), Bp * n_pad, B, n_pad, net0.n_out,
                  _lib.ptr(self.ch_scale), self.scale, self.gate, mean.data_ptr(), est.data_ptr(), flag.data_ptr(),
                  torch.cuda.current_stream().cuda_stream)
        self.launches += 1
        return mean, est, flag.bool()

    def __call__(self, sd: SpectralData, profiles: ProfileBatch, problem: SurrogateProblem,
                 timings: Optional[dict] = None):
        """Channel transmittance [n, n_ch] (device): surrogate where accepted, engine where flagged.

        ``timings`` receives "surrogate_s" and "fallback_s" (synchronised wall times)
        and "n_flagged".
        """
        torch = self.torch
        net0 = self.members[0]
        raw = torch.as_tensor(profiles.features(), device=net0.dev)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        mean, est, flag = self.ensemble(raw)
        flag_h = flag.cpu().numpy()
        t1 = time.perf_counter()
        idx = np.flatnonzero(flag_h)
        if idx.size:
            fb = engine_channels(sd, profiles.subset(idx), problem, as_numpy=False,
                                 deterministic=self.deterministic)
            mean[torch.as_tensor(idx, device=net0.dev)] = fb
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        if timings is not None:
            timings.update({"surrogate_s": t1 - t0, "fallback_s": t2 - t1, "n_flagged": int(idx.size)})
        return mean, est, flag


def calibrate_gate(gs: "GatedSurrogate", raw, reference: np.ndarray, target: float = 1e-3,
                   quantile: float = 0.999, margin: float = 0.5) -> dict:
    """Fit the gate of ``gs`` on a calibration split: ``raw`` features [n, 61] and the
    engine's channel transmittances ``reference`` [n, n_out] of the same profiles (not
    used in training). Tries three per-channel weightings of the members' spread --
    uniform, :func:`channel_weights` of the spread against the ensemble mean's error,
    and its square root -- sets for each the largest threshold that meets the target
    (:func:`gate_threshold`) and keeps the weighting that accepts the most profiles:
    ``gs.ch_scale`` (None for uniform), ``gs.gate`` and ``gs.scale = 1``. Returns the
    fitted values and the split's accepted fraction and accepted-error quantile."""
    torch = gs.torch
    pred = gs.predictions(torch.as_tensor(raw, device=gs.members[0].dev))
    mean = pred.mean(0)
    spread = pred.std(0, unbiased=False).cpu().numpy()
    err_c = np.abs(mean.cpu().numpy() - np.asarray(reference, dtype=np.float32))
    err = err_c.max(1)
    fitted = channel_weights(spread, err_c)
    # candidate weightings; the one whose threshold accepts the most calibration profiles wins
    cands = {"uniform": np.ones_like(fitted), "fitted": fitted, "sqrt_fitted": np.sqrt(fitted).astype(np.float32)}
    trials = {}
    for name, w in cands.items():
        est = (spread * w[None, :]).max(1)
        t = gate_threshold(est, err, target, quantile, margin)
        trials[name] = (float(np.mean(est <= t)), t, est)
    best = max(trials, key=lambda k: trials[k][0])
    acc_frac, t, est = trials[best]
    w = cands[best]
    gs.ch_scale = None if best == "uniform" else torch.as_tensor(w, device=gs.members[0].dev)
    gs.gate, gs.scale = float(t), 1.0
    acc = est <= t
    return {"gate": float(t), "weights": best, "profiles": int(est.size), "accepted": acc_frac,
            "accepted_by_weighting": {k: v[0] for k, v in trials.items()},
            "accepted_err_quantile": float(np.quantile(err[acc], quantile)) if acc.any() else None,
            "spread_vs_error_corr": float(np.corrcoef(est, err)[0, 1]) if est.size > 1 else None,
            "target": target, "quantile": quantile, "margin": margin}


# ---------------------------------------------------------------------------
# Training

@dataclass
class TrainConfig:
    batch: int = 4096
    steps: int = 3000
    lr: float = 1e-3
    lr_final: float = 1e-5
    warmup: int = 100
    seed: int = 0


def lr_at(cfg: TrainConfig, step: int) -> float:
    """Linear warm-up then cosine decay from lr to lr_final."""
    if step < cfg.warmup:
        return cfg.lr * (step + 1) / cfg.warmup
    f = (step - cfg.warmup) / max(1, cfg.steps - cfg.warmup)
    return cfg.lr_final + 0.5 * (cfg.lr - cfg.lr_final) * (1 + math.cos(math.pi * min(f, 1.0)))


class Trainer:
    """Mini-batch Adam over device-resident (features, targets); checkpoint and resume.

    The data order is a seeded permutation per epoch; ``state_dict`` stores the
    network, its optimiser state and the data cursor, so a resumed run continues
    with the same batches and reproduces an uninterrupted run bit for bit.
    """

    def __init__(self, net: MLP, features, targets, cfg: TrainConfig):
        torch = net.torch
        self.net, self.cfg = net, cfg
        self.x = torch.as_tensor(features, dtype=torch.float32, device=net.dev)
        self.y = torch.as_tensor(targets, dtype=torch.float32, device=net.dev)
        if self.x.shape[0] < cfg.batch:
            raise ValueError(f"need at least one batch of samples ({cfg.batch}), got {self.x.shape[0]}")
        self.cursor = 0
        self.epoch = 0
        self._perm = None
        self.losses: List[float] = []

    def _order(self):
        torch = self.net.torch
        if self._perm is None:
            g = torch.Generator().manual_seed(self.cfg.seed * 1_000_003 + self.epoch)
            self._perm = torch.randperm(self.x.shape[0], generator=g).to(self.net.dev)
        return self._perm

    def step(self) -> object:
        cfg = self.cfg
        perm = self._order()
        if self.cursor + cfg.batch > perm.numel():
            self.epoch += 1
            self.cursor = 0
            self._perm = None
            perm = self._order()
        idx = perm[self.cursor:self.cursor + cfg.batch]
        self.cursor += cfg.batch
        return self.net.train_step(self.x[idx], self.y[idx], lr=lr_at(cfg, self.net.step))

    def run(self, steps: Optional[int] = None, log_every: int = 0) -> List[float]:
        n = self.cfg.steps - self.net.step if steps is None else steps
        pending = []
        for i in range(max(0, n)):
            pending.append(self.step())
            if log_every and (self.net.step % log_every == 0):
                self.losses.extend(float(v.item()) for v in pending)
                pending = []
        self.losses.extend(float(v.item()) for v in pending)
        self.net._check(next(iter(self.net._ws.values())))
        return self.losses

    def state_dict(self) -> dict:
        return {"net": self.net.state_dict(), "cursor": self.cursor, "epoch": self.epoch,
                "losses": list(self.losses)}

    def load_state_dict(self, st: dict) -> None:
        self.net.load_state_dict(st["net"])
        self.cursor, self.epoch = int(st["cursor"]), int(st["epoch"])
        self.losses = list(st["losses"])
        self._perm = None


def train_ensemble(features: np.ndarray, targets: np.ndarray, n_members: int = 4, cfg: Optional[TrainConfig] = None,
                   hidden: int = 1024, depth: int = 4) -> List[MLP]:
    """Train ``n_members`` networks that differ in initialisation and data order."""
    cfg = cfg or TrainConfig()
    mean, std = features.mean(0), features.std(0)
    p0 = targets.mean(0)
    members = []
    for m in range(n_members):
        net = MLP(features.shape[1], targets.shape[1], hidden=hidden, depth=depth, seed=cfg.seed * 100 + m)
        net.set_normalisation(mean, std)
        net.set_output_bias(p0)
        tr = Trainer(net, features, targets, TrainConfig(**{**cfg.__dict__, "seed": cfg.seed * 100 + m}))
        tr.run()
        net.train_losses = tr.losses
        members.append(net)
    return members
