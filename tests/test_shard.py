"""Multi-process sharding on CPU: world_size-2 gloo ranks for the profile split + gather
(including a rank with no profiles), the data-parallel gradient all-reduce, and the
wavenumber split's per-rank line restriction (pylblrtm_b200/shard.py)."""

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


def _kept_sorted(nu0, shift, gid, lo_edge, hi_edge, p_max):
    """Host restatement of lbl_sort_lines: kept lines (group, finite centre inside the
    band edges widened by |shift| p_max) sorted by centre, ties by input index."""
    sb = np.abs(shift) * p_max
    keep = (gid >= 0) & np.isfinite(nu0) & (nu0 >= lo_edge - sb) & (nu0 <= hi_edge + sb)
    idx = np.flatnonzero(keep)
    return idx[np.lexsort((idx, nu0[idx]))]


def _tile_candidates(order, nu0, grid, cutoff, pad, tiles):
    """Host restatement of lbl_tile_ranges: each tile's candidate lines (input indices in
    sorted order) whose unshifted centre lies within cutoff + pad of the tile."""
    s = nu0[order]
    out = []
    for t in tiles:
        i0 = t * grid.tile_samples
        i1 = min(i0 + grid.tile_samples, grid.n_nu) - 1
        lo = (grid.nu_at(i0) - cutoff) - pad
        hi = (grid.nu_at(i1) + cutoff) + pad
        out.append(order[np.searchsorted(s, lo, "left"):np.searchsorted(s, hi, "right")])
    return out


def _restriction_matches(world, rank):
    """Rank's shard (its tile span, its line window, the narrowed band edges a shard job
    sorts with) against the full line set: every tile of the span has the same candidate
    lines in the same order, the native host count equals the kept set, and the shard
    keeps fewer lines than the full job."""
    from pylblrtm_b200 import _lib, engine, synthetic
    sd = synthetic.restrict(synthetic.three_gas_lines(40000, 580.0, 720.0, seed=5), 580.0, 720.0)
    lines = {k: v.copy() for k, v in sd.lines.items()}
    lines["shift"] = lines["shift"] * 30.0                # wide pressure shifts stress the pad
    sd = type(sd)(lines, dict(sd.tips), dict(sd.molar_masses), sd.molecule)
    li = engine.layer_input_from_profile(synthetic.logp_profile())
    p_max, cutoff = li.p_max_atm(), 25.0
    grid = engine.make_grid(600.0, 700.0, 0.001, 2.0)
    nu_first, nu_last = grid.nu_at(0), grid.nu_at(grid.n_nu - 1)
    st = {}
    _, gid = engine.select_groups(sd, li.gases, nu_first, nu_last, cutoff, p_max, 3, stats=st)
    pad = st["max_abs_shift"] * p_max * (1 + 1e-9) + 1e-9
    nu0, shift = lines["nu0"].astype(np.float64), lines["shift"].astype(np.float64)
    n_tiles = -(-grid.n_nu // grid.tile_samples)
    span = shard.tile_span(n_tiles, world, rank)
    tiles = range(span.start, span.stop)
    full = _kept_sorted(nu0, shift, gid, *engine.band_edges(nu_first, nu_last, cutoff), p_max)
    win = shard.line_window(sd, grid, cutoff, p_max, span.start, span.stop - span.start)
    lo, hi = engine.band_edges(nu_first, nu_last, cutoff, win)
    part = _kept_sorted(nu0, shift, gid, lo, hi, p_max)
    same = all(np.array_equal(a, b) for a, b in zip(_tile_candidates(full, nu0, grid, cutoff, pad, tiles),
                                                   _tile_candidates(part, nu0, grid, cutoff, pad, tiles)))
    count = _lib.load_host().lbl_count_band(nu0.ctypes.data, shift.ctypes.data, gid.ctypes.data, nu0.size,
                                           lo, hi, p_max)
    return same and count == part.size and (part.size < full.size or world == 1) and len(tiles) > 0


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
        t_lv = rng.uniform(200, 300, (n, 5))
        v = {"H2O": rng.uniform(0, 1e-2, (n, 5))}
        mu = rng.uniform(0.5, 1, n)
        _, full = _fake_batch(None, p, t_lv, v, 1.0, 2.0, mu)
        _, got = shard.transmittance_batch_sharded(None, p, t_lv, v, 1.0, 2.0, mu_view=mu, compute=_fake_batch)
        ok_gather = torch.equal(got, full)
        _, local = shard.transmittance_batch_sharded(None, p, t_lv, v, 1.0, 2.0, mu_view=mu, compute=_fake_batch,
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
        # fewer profiles than ranks: rank 1 computes none and still joins the gather
        _, one = _fake_batch(None, p[:1], t_lv[:1], {"H2O": v["H2O"][:1]}, 1.0, 2.0, mu[:1])
        _, got1 = shard.transmittance_batch_sharded(None, p[:1], t_lv[:1], {"H2O": v["H2O"][:1]}, 1.0, 2.0,
                                                    mu_view=mu[:1], compute=_fake_batch)
        ok_small = torch.equal(got1, one)
        ok_lines = _restriction_matches(world, rank)
        out[rank] = (int(ok_gather) + 2 * int(ok_local) + 4 * int(ok_reduce) + 8 * int(ok_wave) +
                     16 * int(ok_small) + 32 * int(ok_lines))
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
    assert dict(out) == {0: 63, 1: 63}


def test_line_restriction_single_process():
    """The same restriction checks with one rank (the window then spans the whole grid)
    and with four ranks evaluated one after another in this process."""
    assert _restriction_matches(1, 0)
    assert all(_restriction_matches(4, r) for r in range(4))


def test_single_process_is_identity():
    g = [torch.ones(3)]
    shard.allreduce_gradients(g)
    assert torch.equal(g[0], torch.ones(3))
    x = torch.arange(4.0)[:, None]
    assert shard.gather_rows(x, 4) is x
