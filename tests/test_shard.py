"""Multi-process sharding on CPU: world_size-2 gloo ranks for the profile split + gather
and the data-parallel gradient all-reduce (pylblrtm_b200/shard.py)."""

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from pylblrtm_b200 import shard


def test_profile_slice_partitions_exactly():
    for n in (0, 1, 5, 8, 1001):
        for world in (1, 2, 3, 8):
            parts = [shard.profile_slice(n, world, r) for r in range(world)]
            covered = np.concatenate([np.arange(n)[p] for p in parts]) if n else np.array([])
            assert np.array_equal(covered, np.arange(n))
            sizes = [p.stop - p.start for p in parts]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard.profile_slice(4, 2, 2)


def _fake_batch(sd, p, t, v, lo, hi, mu_view, **kw):
    """Stands in for transmittance_batch: one row per profile, depends on its inputs."""
    row = torch.as_tensor(t.sum(1) + 10 * v["H2O"].sum(1) + mu_view, dtype=torch.float64)
    return np.array([lo, hi]), row[:, None] * torch.arange(1, 4, dtype=torch.float64)[None, :]


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rng = np.random.default_rng(0)                 # same inputs on every rank
        n = 7
        p = np.tile(np.linspace(1, 1000, 5), (n, 1))
        t = rng.uniform(200, 300, (n, 5))
        v = {"H2O": rng.uniform(0, 1e-2, (n, 5))}
        mu = rng.uniform(0.5, 1, n)
        _, full = _fake_batch(None, p, t, v, 1.0, 2.0, mu)
        _, got = shard.transmittance_batch_sharded(None, p, t, v, 1.0, 2.0, mu_view=mu, compute=_fake_batch)
        ok_gather = torch.equal(got, full)
        _, local = shard.transmittance_batch_sharded(None, p, t, v, 1.0, 2.0, mu_view=mu, compute=_fake_batch,
                                                     gather=False)
        ok_local = torch.equal(local, full[shard.profile_slice(n, world, rank)])
        # gradient all-reduce: rank r holds (r + 1) * base
        base = [torch.arange(6, dtype=torch.float32).reshape(2, 3), torch.ones(4)]
        grads = [(rank + 1) * g.clone() for g in base]
        shard.allreduce_gradients(grads)
        tot = sum(r + 1 for r in range(world))
        ok_reduce = all(torch.equal(g, tot * b) for g, b in zip(grads, base))
        # wavenumber shards: the fake computation returns each point's global index
        grid_n = 2001                                   # 0.0005 step over 1 cm^-1, tiles of 400 points
        def fake(first, count):
            return torch.arange(first * 400, min(grid_n, (first + count) * 400), dtype=torch.float64)
        nu, t = shard.compute_transmittance_sharded(None, None, 700.0, 701.0, step_cm1=0.0005, tile_width_cm1=0.2,
                                                    compute=fake)
        ok_wave = t.shape == (grid_n,) and np.array_equal(t, np.arange(grid_n, dtype=np.float64)) and nu.size == grid_n
        out[rank] = int(ok_gather) + 2 * int(ok_local) + 4 * int(ok_reduce) + 8 * int(ok_wave)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_gather_and_reduce():
    world = 2
    out = mp.get_context("spawn").Manager().dict()
    mp.start_processes(_worker, args=(world, _free_port(), out), nprocs=world, join=True, start_method="spawn")
    assert dict(out) == {0: 15, 1: 15}


def test_single_process_is_identity():
    g = [torch.ones(3)]
    shard.allreduce_gradients(g)
    assert torch.equal(g[0], torch.ones(3))
    x = torch.arange(4.0)[:, None]
    assert shard.gather_rows(x, 4) is x
