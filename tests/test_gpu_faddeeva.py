"""Device Faddeeva kernels (lbl_faddeeva_f64 / _f32) against scipy.special.wofz."""

import numpy as np
import pytest
from scipy.special import dawsn, erfcx, wofz

from pylblrtm_b200 import _lib

pytestmark = pytest.mark.gpu


def _dev(cuda, x, y, prec, mode=0):
    import torch
    dt = torch.float64 if prec == 64 else torch.float32
    xd = torch.tensor(x, dtype=dt, device=cuda)
    yd = torch.tensor(y, dtype=dt, device=cuda)
    re, im = torch.empty_like(xd), torch.empty_like(xd)
    s = torch.cuda.current_stream().cuda_stream
    if prec == 64:
        _lib.call("lbl_faddeeva_f64", xd.data_ptr(), yd.data_ptr(), xd.numel(), re.data_ptr(), im.data_ptr(), s)
    else:
        _lib.call("lbl_faddeeva_f32", xd.data_ptr(), yd.data_ptr(), xd.numel(), re.data_ptr(), im.data_ptr(),
                  mode, s)
    torch.cuda.synchronize()
    return re.cpu().numpy(), im.cpu().numpy()


def _args(n=100000, seed=0):
    rng = np.random.default_rng(seed)
    x = np.concatenate([rng.uniform(-8, 8, n), np.sign(rng.uniform(-1, 1, n)) * 10 ** rng.uniform(-6, 5, n),
                        rng.uniform(3, 7, n)])
    y = np.concatenate([rng.uniform(0, 6, n), 10 ** rng.uniform(-8, 4, n), 10 ** rng.uniform(-3, 0, n)])
    return x, y


def test_known_answers_f64(cuda):
    re, im = _dev(cuda, [0.0], [0.0], 64)
    assert re[0] == pytest.approx(1.0, abs=1e-15) and im[0] == pytest.approx(0.0, abs=1e-15)
    y = 10 ** np.linspace(-6, 4, 300)
    re, _ = _dev(cuda, np.zeros_like(y), y, 64)
    np.testing.assert_allclose(re, erfcx(y), rtol=1e-11)
    x = np.linspace(-30, 30, 601)
    _, im = _dev(cuda, x, np.zeros_like(x), 64)
    np.testing.assert_allclose(im, 2 / np.sqrt(np.pi) * dawsn(x), rtol=1e-11, atol=1e-300)


def test_dense_grid_f64(cuda):
    x, y = _args()
    ref = wofz(x + 1j * y)
    re, im = _dev(cuda, x, y, 64)
    w = re + 1j * im
    assert np.max(np.abs(w - ref) / np.abs(ref)) < 1e-10
    m = y > 1e-3
    assert np.max(np.abs(re - ref.real)[m] / np.abs(ref.real[m])) < 1e-7


def test_engine_real_part_f32(cuda):
    x, y = _args(seed=3)
    x32, y32 = x.astype(np.float32), y.astype(np.float32)
    ref = wofz(x32.astype(np.float64) + 1j * y32.astype(np.float64)).real
    re, _ = _dev(cuda, x32, y32, 32, mode=1)
    e = np.abs(re - ref) / np.abs(ref)
    assert np.max(e[y32 > 1e-4]) < 2e-6
