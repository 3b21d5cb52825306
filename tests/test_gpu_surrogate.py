"""Surrogate network on the device: the tcgen05 GEMM and its epilogues against torch
float64, the training step's gradients and Adam update against the CPU oracle
(oracle/mlp_ref.py), checkpoint/resume, the ensemble gate, and the trained gated
surrogate against the engine it replaces."""

import ctypes
import time

import numpy as np
import pytest
import torch

from oracle import mlp_ref
from pylblrtm_b200 import _lib, surrogate, synthetic

pytestmark = pytest.mark.gpu


def _bf(shape, gen, scale=1.0):
    return (torch.randn(shape, generator=gen) * scale).to(torch.bfloat16).cuda()


def _gemm(a, b, ep, n_split=1):
    ma, mb = surrogate._Map(a), surrogate._Map(b)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    _lib.call("lbl_gemm_bf16", ma.addr, mb.addr, a.shape[0], b.shape[0], a.shape[1], n_split,
              ctypes.addressof(ep), err.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert err.item() == 0


def _ref(a, b):
    return a.double() @ b.double().T


def _tol(a, b):
    """Bound on the tensor cores' float32 accumulation error: 2^-16 * sum_k |a_k b_k| per
    output (a layout or descriptor error is O(1) of that sum)."""
    return 2.0 ** -16 * (a.double().abs() @ b.double().abs().T) + 1e-30


@pytest.mark.parametrize("m,n,k,split", [(128, 128, 64, 1), (256, 384, 512, 1), (384, 256, 1024, 4),
                                         (1024, 1024, 1024, 2),
                                         # more tiles than SMs: each persistent CTA reuses both accumulators
                                         (4096, 2048, 512, 1), (8192, 384, 256, 1), (38400, 256, 128, 1),
                                         (1024, 1024, 4096, 8)])
def test_gemm_f32_matches_float64(cuda, m, n, k, split):
    g = torch.Generator().manual_seed(m + n + k)
    a, b = _bf((m, k), g), _bf((n, k), g)
    out = torch.full((split, m, n), float("nan"), device="cuda")
    ep = _lib.GemmEpilogue(mode=_lib.GEMM_F32, out_f32=out.data_ptr(), ld_f32=n, split_stride=m * n)
    _gemm(a, b, ep, split)
    got = out.double().sum(0)
    ratio = (torch.abs(got - _ref(a, b)) / _tol(a, b)).max().item()
    assert ratio <= split, ratio


def _close(got, exact, atol, rel=2.0 ** -8):
    """|got - exact| <= rel * |exact| + atol elementwise (rel = half a bf16 ulp by default)."""
    got, exact = got.double(), exact.double()
    return bool(torch.all(torch.abs(got - exact) <= rel * exact.abs() + atol))


def test_gemm_bias_gelu_epilogue(cuda):
    g = torch.Generator().manual_seed(11)
    m, n, k = 256, 256, 256
    a, b = _bf((m, k), g), _bf((n, k), g, 1 / 16)
    bias = torch.randn(n, generator=g).cuda()
    z = torch.empty((m, n), dtype=torch.bfloat16, device="cuda")
    y = torch.empty_like(z)
    yt = torch.empty((n, m), dtype=torch.bfloat16, device="cuda")
    ep = _lib.GemmEpilogue(mode=_lib.GEMM_BIAS_GELU, bias=bias.data_ptr(), z_out=z.data_ptr(), ld_z=n,
                           y=y.data_ptr(), ld_y=n, y_t=yt.data_ptr(), ld_yt=m)
    _gemm(a, b, ep)
    zr = _ref(a, b) + bias.double()
    tol = _tol(a, b)
    assert _close(z, zr, tol)
    assert _close(y, torch.nn.functional.gelu(zr), 1.2 * tol + 1e-6)     # |gelu'| <= 1.13
    assert torch.equal(yt, y.T)


def test_gemm_sigmoid_loss_epilogue(cuda):
    g = torch.Generator().manual_seed(12)
    m, n, k, n_valid = 256, 256, 128, 200
    a, b = _bf((m, k), g), _bf((n, k), g, 1 / 8)
    bias = torch.randn(n, generator=g).cuda()
    target = torch.rand((m, n_valid), generator=g).cuda()
    p = torch.empty((m, n), device="cuda")
    dz = torch.empty((m, n), dtype=torch.bfloat16, device="cuda")
    dzt = torch.empty((n, m), dtype=torch.bfloat16, device="cuda")
    loss = torch.zeros(1, dtype=torch.float64, device="cuda")
    ep = _lib.GemmEpilogue(mode=_lib.GEMM_BIAS_SIGMOID, n_valid=n_valid, bias=bias.data_ptr(), out_f32=p.data_ptr(),
                           ld_f32=n, target=target.data_ptr(), ld_target=n_valid, grad_scale=0.5,
                           y=dz.data_ptr(), ld_y=n, y_t=dzt.data_ptr(), ld_yt=m, loss=loss.data_ptr())
    _gemm(a, b, ep)
    pr = torch.sigmoid(_ref(a, b) + bias.double())
    tol = _tol(a, b)
    assert _close(p, pr, 0.25 * tol + 1e-6, rel=2e-6)                    # sigmoid' <= 1/4
    d = pr[:, :n_valid] - target.double()
    assert abs(loss.item() - (d * d).sum().item()) <= 1e-4 * (d * d).sum().item()
    want = 0.5 * 2 * d * pr[:, :n_valid] * (1 - pr[:, :n_valid])
    assert _close(dz[:, :n_valid], want, 0.5 * tol[:, :n_valid] + 1e-6)  # |d/dz (p - t) p (1 - p)| < 1/2
    assert torch.count_nonzero(dz[:, n_valid:]) == 0
    assert torch.equal(dzt, dz.T)


def test_gemm_dgelu_epilogue(cuda):
    g = torch.Generator().manual_seed(13)
    m, n, k = 128, 256, 384
    a, b = _bf((m, k), g, 1 / 4), _bf((n, k), g, 1 / 4)
    zin = _bf((m, n), g)
    dz = torch.empty((m, n), dtype=torch.bfloat16, device="cuda")
    dzt = torch.empty((n, m), dtype=torch.bfloat16, device="cuda")
    ep = _lib.GemmEpilogue(mode=_lib.GEMM_DGELU, z_in=zin.data_ptr(), ld_zin=n, y=dz.data_ptr(), ld_y=n,
                           y_t=dzt.data_ptr(), ld_yt=m)
    _gemm(a, b, ep)
    gp = torch.from_numpy(mlp_ref.gelu_grad(zin.double().cpu().numpy())).cuda()
    assert _close(dz, _ref(a, b) * gp, 1.2 * _tol(a, b) + 1e-6)
    assert torch.equal(dzt, dz.T)


def test_gemm_argument_errors(cuda):
    a = torch.zeros((128, 64), dtype=torch.bfloat16, device="cuda")
    ma = surrogate._Map(a)
    ep = _lib.GemmEpilogue(mode=_lib.GEMM_F32)
    with pytest.raises(RuntimeError, match="epilogue buffers"):
        _lib.call("lbl_gemm_bf16", ma.addr, ma.addr, 128, 128, 64, 1, ctypes.addressof(ep), 0, 0)
    with pytest.raises(RuntimeError, match="multiples of 128"):
        _lib.call("lbl_gemm_bf16", ma.addr, ma.addr, 100, 128, 64, 1, ctypes.addressof(ep), 0, 0)
    with pytest.raises(RuntimeError, match="rows must be a multiple of 128"):
        surrogate._Map(torch.zeros((100, 64), dtype=torch.bfloat16, device="cuda"))


def _small_net(seed=5):
    net = surrogate.MLP(61, 200, hidden=256, depth=2, seed=seed)
    rng = np.random.default_rng(seed)
    raw = rng.standard_normal((256, 61)).astype(np.float32) * 3 + 1
    target = rng.uniform(0, 1, (256, 200)).astype(np.float32)
    net.set_normalisation(raw.mean(0), raw.std(0))
    net.set_output_bias(target.mean(0))
    return net, raw, target


def _host_params(net):
    w = [t[:nr, :kr].cpu().numpy() for t, (kr, nr) in zip(net.w, net.real)]
    b = [t[:nr].cpu().numpy() for t, (_, nr) in zip(net.b, net.real)]
    return w, b


def test_training_gradients_match_oracle(cuda):
    net, raw, target = _small_net()
    w, b = _host_params(net)
    loss, dw, db = net.gradients(torch.from_numpy(raw).cuda(), torch.from_numpy(target).cuda())
    sse, p, dw_ref, db_ref = mlp_ref.forward_backward(raw, target, net.mean.cpu().numpy(), net.inv_std.cpu().numpy(),
                                                      w, b, grad_scale=1.0 / 256)
    assert abs(loss - sse / (256 * 200)) <= 1e-5 * sse / (256 * 200)
    for l in range(len(dw)):
        g, r = dw[l].double().cpu().numpy(), dw_ref[l]
        assert np.linalg.norm(g - r) <= 2e-3 * np.linalg.norm(r), l
        g, r = db[l].double().cpu().numpy(), db_ref[l]
        assert np.linalg.norm(g - r) <= 2e-3 * np.linalg.norm(r), l
    # inference output = the oracle's sigmoid output
    out = net.predict(torch.from_numpy(raw).cuda()).double().cpu().numpy()
    assert np.max(np.abs(out - p)) < 2e-5


def test_data_parallel_gradient_scaling(cuda):
    """Two ranks of 128 with scale 1/(128 x 2) sum to the 256-row batch gradient (what
    shard.allreduce_gradients computes between backward and Adam)."""
    net, raw, target = _small_net(7)
    r, t = torch.from_numpy(raw).cuda(), torch.from_numpy(target).cuda()
    _, dw, db = net.gradients(r, t)
    net.world = 2
    try:
        _, dw_a, db_a = net.gradients(r[:128], t[:128])
        _, dw_b, db_b = net.gradients(r[128:], t[128:])
    finally:
        net.world = 1
    for full, a, b in zip(dw + db, dw_a + db_a, dw_b + db_b):
        assert torch.linalg.norm(a + b - full) <= 1e-5 * torch.linalg.norm(full)


def test_adam_step_matches_oracle(cuda):
    net, raw, target = _small_net(6)
    w0, b0 = _host_params(net)
    _, dw, db = net.gradients(torch.from_numpy(raw).cuda(), torch.from_numpy(target).cuda())
    ws = net.workspace(256, True)
    net._adam(ws, torch.cuda.current_stream().cuda_stream, 1e-3)
    w1, b1 = _host_params(net)
    for l in range(len(w0)):
        wr, _, _ = mlp_ref.adam(w0[l], 0 * w0[l], 0 * w0[l], dw[l].cpu().numpy(), 1, 1e-3)
        np.testing.assert_allclose(w1[l], wr, rtol=0, atol=1e-7)
        br, _, _ = mlp_ref.adam(b0[l], 0 * b0[l], 0 * b0[l], db[l].cpu().numpy(), 1, 1e-3)
        np.testing.assert_allclose(b1[l], br, rtol=0, atol=1e-7)
        assert torch.equal(net.w_bf[l], net.w[l].to(torch.bfloat16))
        assert torch.equal(net.wt_bf[l], net.w[l].T.to(torch.bfloat16))


def _toy_data(n, seed=0):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((n, 61)).astype(np.float32)
    a = rng.standard_normal((61, 200)) / 8
    y = 1 / (1 + np.exp(-np.sin(x @ a) * 2))
    return x, y.astype(np.float32)


def test_training_reduces_loss_and_resume_is_exact(cuda):
    x, y = _toy_data(4096)
    cfg = surrogate.TrainConfig(batch=512, steps=300, lr=2e-3, warmup=20, seed=3)

    def fresh():
        net = surrogate.MLP(61, 200, hidden=256, depth=2, seed=1)
        net.set_normalisation(x.mean(0), x.std(0))
        net.set_output_bias(y.mean(0))
        return net, surrogate.Trainer(net, x, y, cfg)

    net, tr = fresh()
    tr.run(40)
    ck = tr.state_dict()
    tr.run()
    losses = tr.losses
    assert np.mean(losses[-20:]) < 0.25 * np.mean(losses[:5])
    net2, tr2 = fresh()
    tr2.load_state_dict(ck)
    tr2.run()
    for a, b in zip(net.w, net2.w):
        assert torch.equal(a, b)
    assert tr2.losses[-10:] == losses[-10:]


def test_ensemble_gate_matches_numpy(cuda):
    g = torch.Generator().manual_seed(4)
    n_mem, B, ld, n_ch = 4, 300, 256, 200
    pred = torch.rand((n_mem, B, ld), generator=g).cuda()
    pred[:, :150] = pred[0:1, :150] + 1e-4 * pred[:, :150]       # tight members for half the samples
    mean = torch.empty((B, n_ch), device="cuda")
    est = torch.empty(B, device="cuda")
    flag = torch.empty(B, dtype=torch.int32, device="cuda")
    _lib.call("lbl_ensemble_gate", pred.data_ptr(), n_mem, B * ld, B, ld, n_ch, 0, 2.0, 1e-3, mean.data_ptr(),
              est.data_ptr(), flag.data_ptr(), 0)
    torch.cuda.synchronize()
    p = pred[:, :, :n_ch].double().cpu().numpy()
    np.testing.assert_allclose(mean.cpu().numpy(), p.mean(0), rtol=1e-6)
    np.testing.assert_allclose(est.cpu().numpy(), p.std(0).max(1), rtol=1e-3, atol=1e-7)
    np.testing.assert_array_equal(flag.cpu().numpy(), (2.0 * est.cpu().numpy() > 1e-3).astype(np.int32))
    assert flag[:150].sum() == 0 and flag[150:].sum() == 150
    # per-channel weights (a calibrated gate): est = max_c w_c std_c
    w = torch.rand(n_ch, generator=g) * 3.0
    _lib.call("lbl_ensemble_gate", pred.data_ptr(), n_mem, B * ld, B, ld, n_ch, w.cuda().data_ptr(), 1.0, 0.5,
              mean.data_ptr(), est.data_ptr(), flag.data_ptr(), 0)
    torch.cuda.synchronize()
    ref = (p.std(0) * w.double().numpy()[None, :]).max(1)
    np.testing.assert_allclose(est.cpu().numpy(), ref, rtol=1e-3, atol=1e-7)
    np.testing.assert_array_equal(flag.cpu().numpy(), (est.cpu().numpy() > 0.5).astype(np.int32))


def test_gated_surrogate_against_engine(cuda):
    """A small trained surrogate: accurate in distribution, OOD flagged, fallback exact, and faster."""
    problem = surrogate.SurrogateProblem(nu_min=700.0, nu_max=720.0, step=0.001, channel_width=0.25)
    # 1/10 of the 200k-line density with strengths x 1e-3: channel T spans ~0.08-0.8
    # (at full strength every channel of this window is saturated, T < 1e-10)
    sd = synthetic.scale_strengths(synthetic.restrict(synthetic.three_gas_lines(20_000), 675.0, 745.0), 1e-3)
    train = surrogate.sample_profiles(4096, seed=1)
    x = train.features()
    y = surrogate.engine_channels(sd, train, problem, profiles_per_launch=256)
    members = surrogate.train_ensemble(x, y, n_members=4, hidden=256, depth=2,
                                       cfg=surrogate.TrainConfig(batch=512, steps=600, lr=2e-3, warmup=30, seed=7))
    test_in = surrogate.sample_profiles(512, seed=2)
    test_ood = surrogate.sample_profiles(512, seed=3, t_offset=25.0)
    gate = surrogate.GatedSurrogate(members, deterministic=True)
    ref_in = surrogate.engine_channels(sd, test_in, problem, deterministic=True)
    ref_ood = surrogate.engine_channels(sd, test_ood, problem, deterministic=True)
    mean_in, est_in, _ = gate.ensemble(torch.from_numpy(test_in.features()).cuda())
    gate.gate = float(np.quantile(est_in.cpu().numpy(), 0.9))      # 10 % of in-distribution flagged
    _, est_ood, flag_ood = gate.ensemble(torch.from_numpy(test_ood.features()).cuda())
    err_in = np.abs(mean_in.cpu().numpy() - ref_in).max(1)
    # in distribution the surrogate is far better than the best input-independent guess
    base = np.abs(y.mean(0)[None] - ref_in).max(1)
    assert np.median(err_in) < 0.1 * np.median(base)
    # out of distribution the ensemble disagrees more
    assert np.median(est_ood.cpu().numpy()) > 2 * np.median(est_in.cpu().numpy())
    assert flag_ood.float().mean() > 0.2
    # the gated result equals the engine wherever it fell back
    t = {}
    out, _, flag = gate(sd, test_ood, problem, timings=t)
    fb = flag.cpu().numpy()
    assert fb.any()
    np.testing.assert_array_equal(out.cpu().numpy()[fb], ref_ood[fb].astype(np.float32))
    # speed: surrogate-only evaluation against the engine on the same 512 profiles
    raw = torch.from_numpy(test_in.features()).cuda()
    gate.ensemble(raw)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    gate.ensemble(raw)
    torch.cuda.synchronize()
    t_sur = time.perf_counter() - t0
    t0 = time.perf_counter()
    surrogate.engine_channels(sd, test_in, problem, profiles_per_launch=512)
    torch.cuda.synchronize()
    t_eng = time.perf_counter() - t0
    assert t_eng > 5 * t_sur, (t_eng, t_sur)
    # calibration on a split of its own: weights and threshold such that the accepted
    # calibration profiles meet a target; on fresh profiles the accepted error quantile
    # stays near it (the calibration split and the test set are different draws)
    cal = surrogate.sample_profiles(2048, seed=4)
    ref_cal = surrogate.engine_channels(sd, cal, problem, deterministic=True)
    target = float(np.quantile(err_in, 0.7))
    fit = surrogate.calibrate_gate(gate, cal.features(), ref_cal, target=target, quantile=0.95, margin=0.5)
    assert fit["weights"] in ("uniform", "fitted", "sqrt_fitted")
    assert fit["accepted"] == max(fit["accepted_by_weighting"].values())
    assert (gate.ch_scale is None) == (fit["weights"] == "uniform")
    assert gate.ch_scale is None or gate.ch_scale.shape == (problem.n_channels,)
    assert 0.0 < fit["accepted"] < 1.0 and fit["accepted_err_quantile"] <= target
    mean2, est2, flag2 = gate.ensemble(torch.from_numpy(test_in.features()).cuda())
    acc = ~flag2.cpu().numpy()
    err2 = np.abs(mean2.cpu().numpy() - ref_in).max(1)
    assert acc.any() and np.quantile(err2[acc], 0.95) <= 1.5 * target
    flag_ood2 = gate.ensemble(torch.from_numpy(test_ood.features()).cuda())[2].cpu().numpy()
    assert flag_ood2.mean() > flag2.cpu().numpy().mean()
