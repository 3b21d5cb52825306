"""The allocation-free line sort (lbl_sort_lines_noalloc) against lbl_sort_lines.

lbl_sort_lines_noalloc serves callers that cannot allocate device memory when
they run: its scratch is a static array inside the library instead of a
workspace passed in by the caller. This file is collected last so that a run
stopping at the first failure has already run every other test; it also passes
on its own in a fresh process.
"""

import numpy as np
import pytest

from pylblrtm_b200 import _lib

pytestmark = pytest.mark.gpu


def _inputs(seed, n):
    rng = np.random.default_rng(seed)
    nu0 = rng.uniform(500.0, 2600.0, n)               # some lines fall outside the band mask
    nu0[rng.integers(0, n, n // 50)] = 1000.0          # ties, broken by input index
    shift = rng.uniform(-0.004, 0.0, n)
    gid = rng.integers(-1, 3, n).astype(np.int32)      # -1 drops a line
    return nu0, shift, gid


def _sort(cuda, fn, nu0, shift, gid):
    import torch
    n = nu0.size
    d_nu0 = torch.tensor(nu0, device=cuda)
    d_shift = torch.tensor(shift, device=cuda)
    d_gid = torch.tensor(gid, device=cuda)
    order = torch.full((n,), -7, dtype=torch.int32, device=cuda)
    kept = torch.full((1,), -7, dtype=torch.int32, device=cuda)
    sb = torch.full((1,), -7.0, dtype=torch.float64, device=cuda)
    stream = torch.cuda.current_stream().cuda_stream
    args = (d_nu0.data_ptr(), d_shift.data_ptr(), d_gid.data_ptr(), n, 600.0 - 25.0, 2500.0 + 25.0, 1.0)
    if fn == "lbl_sort_lines":
        ws_bytes = _lib.load().lbl_sort_workspace_bytes(n)
        ws = torch.empty((ws_bytes + 7) // 8, dtype=torch.float64, device=cuda)
        _lib.call(fn, *args, ws.data_ptr(), ws_bytes, order.data_ptr(), kept.data_ptr(), sb.data_ptr(), stream)
    else:
        _lib.call(fn, *args, order.data_ptr(), kept.data_ptr(), sb.data_ptr(), stream)
    torch.cuda.synchronize()
    k = int(kept.item())
    return order.cpu().numpy()[:k], k, float(sb.item())


def test_noalloc_sort_matches_workspace_sort_twice(cuda):
    # two calls in a row with different inputs and sizes: the static scratch keeps
    # the previous call's contents, which must not affect the next result
    for seed, n in ((11, 200_000), (12, 3_001)):
        nu0, shift, gid = _inputs(seed, n)
        ref = _sort(cuda, "lbl_sort_lines", nu0, shift, gid)
        got = _sort(cuda, "lbl_sort_lines_noalloc", nu0, shift, gid)
        assert got[1] == ref[1] > 0
        assert np.array_equal(got[0], ref[0])
        assert got[2] == ref[2]
        keys = nu0[got[0]]
        assert np.all(np.diff(keys) >= 0)


def test_noalloc_sort_rejects_more_lines_than_its_scratch(cuda):
    n = (1 << 18) + 1
    with pytest.raises(RuntimeError, match="exceed the static scratch limit of 262144 lines"):
        _lib.call("lbl_sort_lines_noalloc", 1, 1, 1, n, 0.0, 1.0, 1.0, 1, 1, 1, 0)
