"""Multi-GPU sharding (one process per GPU, ``torch.distributed``).

The forward model shards without any data-path exchange: profiles of a batch are
independent, so each rank computes a contiguous slice of them
(:func:`profile_slice`) and the results are gathered once at the end
(:func:`transmittance_batch_sharded`, an all-gather over NCCL / NVLink, or over gloo
on CPU). A single spectrum is not split: every rank runs its own (the bench's
replicas, weak scaling).

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
