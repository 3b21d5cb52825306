"""Accuracy of the engine's Faddeeva routines (host build of faddeeva.cuh) against scipy.special.wofz."""

import ctypes
import os

import numpy as np
import pytest
from scipy.special import dawsn, erfcx, wofz

from conftest import ROOT

LIB = os.path.join(ROOT, "pylblrtm_b200", "libfaddeeva_host.so")


@pytest.fixture(scope="module")
def host():
    lib = ctypes.CDLL(LIB)
    P, L, I = ctypes.c_void_p, ctypes.c_longlong, ctypes.c_int
    lib.lbl_host_faddeeva_f64.argtypes = [P, P, L, P, P]
    lib.lbl_host_faddeeva_f32.argtypes = [P, P, L, P, P, I]

    def f64(x, y):
        x = np.ascontiguousarray(x, np.float64)
        y = np.ascontiguousarray(y, np.float64)
        re, im = np.empty_like(x), np.empty_like(x)
        lib.lbl_host_faddeeva_f64(x.ctypes.data, y.ctypes.data, x.size, re.ctypes.data, im.ctypes.data)
        return re + 1j * im

    def f32(x, y, mode):
        x = np.ascontiguousarray(x, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        re, im = np.empty_like(x), np.empty_like(x)
        lib.lbl_host_faddeeva_f32(x.ctypes.data, y.ctypes.data, x.size, re.ctypes.data, im.ctypes.data, mode)
        return re, im
    return f64, f32


def _args(n=60000, seed=0):
    rng = np.random.default_rng(seed)
    x = np.concatenate([rng.uniform(-8, 8, n), np.sign(rng.uniform(-1, 1, n)) * 10 ** rng.uniform(-6, 5, n),
                        rng.uniform(3, 7, n)])
    y = np.concatenate([rng.uniform(0, 6, n), 10 ** rng.uniform(-8, 4, n), 10 ** rng.uniform(-3, 0, n)])
    return x, y


def test_f64_known_answers(host):
    f64, _ = host
    assert f64(np.array([0.0]), np.array([0.0]))[0] == pytest.approx(1.0, abs=1e-15)
    y = 10 ** np.linspace(-6, 4, 200)
    np.testing.assert_allclose(f64(np.zeros_like(y), y).real, erfcx(y), rtol=1e-11)
    x = np.linspace(-30, 30, 601)
    np.testing.assert_allclose(f64(x, np.zeros_like(x)).imag, 2 / np.sqrt(np.pi) * dawsn(x), rtol=1e-11,
                               atol=1e-300)


def test_f64_against_wofz(host):
    f64, _ = host
    x, y = _args()
    ref = wofz(x + 1j * y)
    w = f64(x, y)
    assert np.max(np.abs(w - ref) / np.abs(ref)) < 1e-10
    m = y > 1e-3
    assert np.max(np.abs(w.real - ref.real)[m] / np.abs(ref.real[m])) < 1e-7
    # lower half plane through the reflection formula
    rng = np.random.default_rng(1)
    xn, yn = rng.uniform(-4, 4, 20000), -rng.uniform(0, 3, 20000)
    refn = wofz(xn + 1j * yn)
    assert np.max(np.abs(f64(xn, yn) - refn) / np.abs(refn)) < 1e-10


def test_f32_engine_real_part(host):
    """The float32 engine's Re w (mode 1) is within 2e-6 relative for every region."""
    _, f32 = host
    x, y = _args(seed=2)
    x32, y32 = x.astype(np.float32), y.astype(np.float32)
    ref = wofz(x32.astype(np.float64) + 1j * y32.astype(np.float64)).real
    re, _ = f32(x32, y32, 1)
    e = np.abs(re - ref) / np.abs(ref)
    assert np.max(e[y32 > 1e-4]) < 2e-6, np.max(e[y32 > 1e-4])


def test_eight_term_series_on_the_near_zone_tails(host):
    """The near-zone tails (36 <= |z|^2 < 64) of the float32 multi-level engine take eight terms
    of the asymptotic series (mode 2): Re w within 5e-7 relative for y from 1e-4 to 6, as the
    float continued fraction it replaced, with no loss of relative accuracy for small y."""
    _, f32 = host
    rng = np.random.default_rng(3)
    y = np.concatenate([10 ** rng.uniform(-4, 0, 20000), rng.uniform(1, 6, 20000)])
    r = np.sqrt(rng.uniform(36.0, 64.0, y.size))
    ok = r > y
    y, r = y[ok], r[ok]
    x = np.sqrt(r * r - y * y) * np.sign(rng.uniform(-1, 1, y.size))
    re, _ = f32(x, y, 2)
    xf, yf = x.astype(np.float32).astype(np.float64), y.astype(np.float32).astype(np.float64)
    z2 = xf * xf + yf * yf
    band = (z2 >= 36.0) & (z2 < 64.0)
    ref = wofz(xf + 1j * yf).real
    assert np.max(np.abs(re[band] - ref[band]) / ref[band]) <= 5e-7


def test_weideman_coefficient_sets():
    """Both Weideman sets of weideman_coeffs.h inside |z|^2 < 36 (where the engines use
    them) against wofz: the 36-term set to 2e-14 of |w|, the float32 engine's 28-term set
    to 7e-7 of Re w for y >= 1e-4 and 1e-8 of Re w for y >= 0.01."""
    lib = ctypes.CDLL(LIB)
    P = ctypes.c_void_p
    lib.lbl_host_weideman_re.argtypes = [P, P, ctypes.c_longlong, ctypes.c_int, P]
    x1 = np.linspace(-6, 6, 1201)
    for ymin, bound28 in ((1e-4, 7e-7), (1e-2, 1e-8)):
        X, Y = np.meshgrid(x1, np.geomspace(ymin, 6, 120))
        m = X ** 2 + Y ** 2 < 36
        x, y = np.ascontiguousarray(X[m]), np.ascontiguousarray(Y[m])
        ref = wofz(x + 1j * y)
        for terms in (36, 28):
            re = np.empty_like(x)
            assert lib.lbl_host_weideman_re(x.ctypes.data, y.ctypes.data, x.size, terms, re.ctypes.data) == 0
            rel = np.max(np.abs(re - ref.real) / np.abs(ref.real))
            if terms == 28:
                assert rel <= bound28, (ymin, rel)
            else:
                assert np.max(np.abs(re - ref.real) / np.abs(ref)) <= 2e-14
    assert lib.lbl_host_weideman_re(x.ctypes.data, y.ctypes.data, 1, 30, re.ctypes.data) == -1
