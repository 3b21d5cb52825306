"""Multi-GPU sharding (one process per GPU, ``torch.distributed``).

The forward model shards without any data-path exchange: profiles of a batch are
independent, so each rank computes a contiguous slice of them
(:func:`profile_slice`; a rank may get none) and the results are gathered once at the
end (:func:`transmittance_batch_sharded`, an all-gather over NCCL / NVLink, or over
gloo on CPU). One spectrum splits by wavenumber (:func:`compute_transmittance_sharded`):
each rank computes a contiguous range of the grid's reference tiles
(:func:`tile_span`) with the grid values of the full grid, from only the lines that
can reach those tiles (:func:`line_window`: the tiles widened by the cut-off and the
largest pressure shift), so line preparation and its memory shrink with the rank
count. The tile-window rule (``pylblrtm/forward.py:295-301``) makes the tiles
independent, every tile sees the same candidate lines in the same order as in the
full job, and the pieces are all-gathered; with the deterministic sums the result
equals the single-GPU spectrum bit for bit.

The surrogate's training has one real exchange step: data-parallel ranks sum their
weight and bias gradients (:func:`allreduce_gradients`) between the backward pass and
the Adam update, each rank having scaled its loss by 1 / (local batch x world) so the
sum is the global-batch mean. Every rank takes the same collective steps in the same
order.
"""

from __future__ import annotations

from typing import Callable, Optional, Sequence

import numpy as np


def _dist():
    import torch.distributed as dist
    return dist


def world_and_rank(group=None):
    dist = _dist()
    if not dist.is_available() or not dist.is_initialized():
        return 1, 0
    return dist.get_world_size(group), dist.get_rank(group)


def profile_slice(n: int, world: int, rank: int) -> slice:
    """Contiguous, balanced share of n profiles for ``rank`` (the first n % world ranks get one more)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("need 0 <= rank < world")
    base, extra = divmod(int(n), world)
    start = rank * base + min(rank, extra)
    return slice(start, start + base + (1 if rank < extra else 0))


def tile_span(n_tiles: int, world: int, rank: int) -> slice:
    """Contiguous share of the reference tiles [0, n_tiles) for ``rank``."""
    return profile_slice(n_tiles, world, rank)


def line_window(spectral_data, grid, cutoff: float, p_max: float, first: int, count: int):
    """Unshifted line centres [lo, hi] that reference tiles [first, first + count) of
    ``grid`` can use: the tiles' first and last grid values widened by the larger of the
    cut-off and the tile width (the summation's inner-line reach), plus the largest
    finite |shift| x p_max and a few grid steps of margin. Every candidate line of those
    tiles (``forward.py:295-301``, unshifted centres within cut-off + shift bound) lies
    inside it."""
    shift = np.abs(np.asarray(spectral_data.lines["shift"], dtype=np.float64))
    shift = shift[np.isfinite(shift)]
    pad = (float(shift.max()) if shift.size else 0.0) * float(p_max) * (1 + 1e-6) + 1e-6
    ts = grid.tile_samples
    i0 = first * ts
    i1 = min(grid.n_nu, (first + count) * ts) - 1
    reach = max(float(cutoff), ts * grid.step) + pad + 8 * grid.step
    return grid.nu_at(i0) - reach, grid.nu_at(i1) + reach


def gather_rows(local, n_total: int, group=None):
    """All-gather row blocks [n_r, ...] of every rank into [n_total, ...] (rank order).

    Blocks are padded to the largest share so one all_gather suffices; the result is
    identical on every rank.
    """
    import torch
    dist = _dist()
    world, _ = world_and_rank(group)
    if world == 1:
        return local
    counts = [profile_slice(n_total, world, r).stop - profile_slice(n_total, world, r).start for r in range(world)]
    m = max(counts)
    pad = torch.zeros((m,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    pad[: local.shape[0]] = local
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad, group=group)
    return torch.cat([p[:c] for p, c in zip(parts, counts)], dim=0)


def transmittance_batch_sharded(spectral_data, pressure_hpa, temperature_k, vmr, nu_min_cm1, nu_max_cm1, *,
                                group=None, gather: bool = True, compute: Optional[Callable] = None, **kwargs):
    """``batch.transmittance_batch`` with the profiles split across the ranks of ``group``.

    Returns ``(axis, T)`` where T holds all profiles (``gather=True``, same on every
    rank) or only this rank's slice; ``compute`` replaces ``transmittance_batch``
    (tests). ``mu_view`` may be per profile; it is sliced like the profiles.
    """
    if compute is None:
        from .batch import transmittance_batch as compute
    p = np.atleast_2d(np.asarray(pressure_hpa, dtype=np.float64))
    n = p.shape[0]
    world, rank = world_and_rank(group)
    sl = profile_slice(n, world, rank)
    t = np.atleast_2d(np.asarray(temperature_k, dtype=np.float64))[sl]
    v = {g: np.atleast_2d(np.asarray(a, dtype=np.float64))[sl] for g, a in vmr.items()}
    mu = kwargs.pop("mu_view", 1.0)
    mu = np.broadcast_to(np.asarray(mu, dtype=np.float64), (n,))[sl]
    kwargs["as_numpy"] = False
    axis, local = compute(spectral_data, p[sl], t, v, nu_min_cm1, nu_max_cm1, mu_view=mu, **kwargs)
    if not gather:
        return axis, local
    return axis, gather_rows(local, n, group)


def gather_pieces(local, counts: Sequence[int], group=None):
    """All-gather 1-D pieces of known lengths ``counts`` (rank order) into one tensor."""
    import torch
    dist = _dist()
    world, _ = world_and_rank(group)
    if world == 1:
        return local
    m = max(max(counts), 1)
    pad = torch.zeros(m, dtype=local.dtype, device=local.device)
    pad[: local.numel()] = local
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad, group=group)
    return torch.cat([p[:c] for p, c in zip(parts, counts)])


def shard_job(spectral_data, profile, grid, cutoff: float, first: int, count: int, warn_level: int = 4):
    """``engine.Job`` of one wavenumber shard: only the lines of :func:`line_window`
    go to the device; group selection and warnings use the whole line list."""
    from . import engine
    li = engine.layer_input_from_profile(profile)
    win = line_window(spectral_data, grid, cutoff, li.p_max_atm(), first, count)
    return engine.Job(spectral_data, li, grid, float(cutoff), warn_level=warn_level, line_window=win)


def compute_transmittance_sharded(spectral_data, profile, nu_min_cm1: float, nu_max_cm1: float, *,
                                  step_cm1: float = 0.001, line_cutoff_cm1: float = 25.0,
                                  tile_width_cm1: float = 2.0, mu_view: float = 1.0, deterministic: bool = True,
                                  group=None, compute: Optional[Callable] = None):
    """``compute_transmittance`` with the reference tiles of the grid split across the
    ranks of ``group`` (multi-level float32 engine); each rank prepares only the lines
    its tiles can use. Every rank returns the full ``(nu, T)``. ``compute(first,
    count)`` replaces the device computation of a tile range (tests); it returns that
    range's transmittance as a 1-D tensor.
    """
    import torch
    from . import engine
    from .atmosphere import AtmosphericProfile
    from .spectral_data import SpectralData
    if compute is None:
        if not isinstance(spectral_data, SpectralData):
            raise TypeError("spectral_data must be a SpectralData instance")
        if not isinstance(profile, AtmosphericProfile):
            raise TypeError("profile must be an AtmosphericProfile instance")
    if nu_min_cm1 >= nu_max_cm1:
        raise ValueError("nu_min_cm1 must be strictly less than nu_max_cm1")
    if step_cm1 <= 0:
        raise ValueError("step_cm1 must be positive")
    if not (0.0 < mu_view <= 1.0):
        raise ValueError("mu_view must be in (0, 1]")
    grid = engine.make_grid(nu_min_cm1, nu_max_cm1, step_cm1, tile_width_cm1)
    ts = grid.tile_samples
    n_tiles = -(-grid.n_nu // ts)
    world, rank = world_and_rank(group)
    spans = [tile_span(n_tiles, world, r) for r in range(world)]
    counts = [max(0, min(grid.n_nu, sl.stop * ts) - sl.start * ts) if sl.stop > sl.start else 0 for sl in spans]
    sl = spans[rank]
    if compute is None:
        def compute(first, count):
            job = shard_job(spectral_data, profile, grid, float(line_cutoff_cm1), first, count, warn_level=3)
            res = job.run("fp32", mu=[float(mu_view)], want_od=False, want_trans=True,
                          deterministic=deterministic, tiles=(first, count))
            return res.trans[0]
    dev = torch.device("cuda", torch.cuda.current_device()) if torch.cuda.is_available() else torch.device("cpu")
    local = compute(sl.start, sl.stop - sl.start) if sl.stop > sl.start else \
        torch.zeros(0, dtype=torch.float64, device=dev)
    full = gather_pieces(local, counts, group)
    out = full.cpu().numpy() if full.is_cuda else full.numpy()
    return grid.nu, out


def allreduce_gradients(grads: Sequence, group=None) -> None:
    """Sum gradient tensors across the ranks of ``group`` in place (one bucket)."""
    import torch
    dist = _dist()
    world, _ = world_and_rank(group)
    if world == 1 or not grads:
        return
    flat = torch.cat([g.reshape(-1) for g in grads])
    dist.all_reduce(flat, op=dist.ReduceOp.SUM, group=group)
    off = 0
    for g in grads:
        k = g.numel()
        g.view(-1).copy_(flat[off:off + k])
        off += k
