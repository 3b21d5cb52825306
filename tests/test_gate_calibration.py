"""Host logic of the surrogate gate's calibration (pylblrtm_b200.surrogate): the
threshold that keeps the accepted profiles' error quantile under the target, and the
per-channel spread weights."""

import numpy as np

from pylblrtm_b200.surrogate import channel_weights, gate_threshold


def test_threshold_meets_the_quantile_target_with_margin():
    rng = np.random.default_rng(0)
    n = 200_000
    err = rng.lognormal(np.log(2.5e-4), 0.6, n)
    est = err * np.exp(rng.normal(0.0, 0.3, n))          # an estimate correlated with the error
    t = gate_threshold(est, err, target=1e-3, quantile=0.999, margin=0.5)
    acc = est <= t
    assert 0.5 < acc.mean() < 1.0
    assert np.mean(err[acc] > 1e-3) <= 0.5 * 1e-3 + 1e-12
    # the largest such threshold: accepting the next profile breaks the rule
    nxt = np.min(est[est > t])
    acc2 = est <= nxt
    assert np.sum(err[acc2] > 1e-3) > 0.5 * 1e-3 * acc2.sum()


def test_threshold_edge_cases():
    est = np.array([1.0, 2.0, 2.0, 3.0])
    assert gate_threshold(est, np.zeros(4)) == 3.0          # nothing bad: accept all
    assert gate_threshold(est, np.ones(4)) == 0.0           # everything bad: accept none
    # ties: a threshold never splits profiles with the same estimate
    err = np.array([0.0, 0.0, 1.0, 0.0])
    assert gate_threshold(est, err, target=0.5, quantile=0.0, margin=0.2) == 1.0


def test_channel_weights_rescale_spread_to_error():
    rng = np.random.default_rng(1)
    spread = rng.uniform(0.5, 1.5, (5000, 8)) * np.array([1, 2, 4, 8, 1, 1, 1, 1.0])
    err = spread * np.array([4, 2, 1, 0.5, 1, 1, 1, 1.0])     # channels' error/spread ratios differ
    w = channel_weights(spread, err)
    assert w.dtype == np.float32 and w.shape == (8,)
    np.testing.assert_allclose(w / w[4], [4, 2, 1, 0.5, 1, 1, 1, 1], rtol=1e-6)
    assert np.isclose(np.median(w), 1.0)
    # degenerate channels (no spread, no error) get weight 1 before normalisation
    w0 = channel_weights(np.zeros((10, 3)), np.zeros((10, 3)))
    np.testing.assert_allclose(w0, 1.0)
