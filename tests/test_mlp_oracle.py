"""The surrogate network's CPU oracle (oracle/mlp_ref.py) against torch: bf16 rounding,
the hand-written backward pass (float64 autograd) and Adam (torch.optim.Adam)."""

import numpy as np
import torch

from oracle import mlp_ref


def test_bf16_rounding_matches_torch():
    rng = np.random.default_rng(0)
    x = np.concatenate([rng.standard_normal(10000).astype(np.float32) * 10.0 ** rng.integers(-8, 8, 10000),
                        # exact ties: 1 + (2k+1) * 2^-8 lie half-way between bf16 neighbours
                        (1.0 + (2 * np.arange(64) + 1) * 2.0 ** -8).astype(np.float32),
                        np.array([0.0, -0.0, 1e-40, -3e38], np.float32)])
    ref = torch.from_numpy(x).to(torch.bfloat16).float().numpy()
    assert np.array_equal(mlp_ref.bf16(x).view(np.uint32), ref.view(np.uint32))


def _net(rng, dims):
    w = [(rng.standard_normal((n, k)) / np.sqrt(k)).astype(np.float32) for k, n in dims]
    b = [(0.1 * rng.standard_normal(n)).astype(np.float32) for _, n in dims]
    return w, b


def test_backward_matches_float64_autograd():
    rng = np.random.default_rng(1)
    dims = [(7, 32), (32, 32), (32, 5)]
    w, b = _net(rng, dims)
    raw = rng.standard_normal((16, 7)).astype(np.float32)
    target = rng.uniform(0, 1, (16, 5))
    mean, inv_std = raw.mean(0), 1.0 / raw.std(0)
    scale = 1.0 / 16
    sse, p, dw, db = mlp_ref.forward_backward(raw, target, mean, inv_std, w, b, scale, rounding=False)

    tw = [torch.tensor(a, dtype=torch.float64, requires_grad=True) for a in w]
    tb = [torch.tensor(a, dtype=torch.float64, requires_grad=True) for a in b]
    x = (torch.tensor(raw, dtype=torch.float64) - torch.tensor(mean, dtype=torch.float64)) * \
        torch.tensor(inv_std, dtype=torch.float64)
    for l in range(len(dims)):
        z = x @ tw[l].T + tb[l]
        x = torch.nn.functional.gelu(z) if l < len(dims) - 1 else torch.sigmoid(z)
    loss = scale * ((x - torch.tensor(target)) ** 2).sum()
    loss.backward()
    assert abs(sse * scale - loss.item()) < 1e-12
    np.testing.assert_allclose(p, x.detach().numpy(), rtol=1e-12)
    for l in range(len(dims)):
        np.testing.assert_allclose(dw[l], tw[l].grad.numpy(), rtol=1e-9, atol=1e-14)
        np.testing.assert_allclose(db[l], tb[l].grad.numpy(), rtol=1e-9, atol=1e-14)


def test_rounded_pass_stays_close_to_exact():
    rng = np.random.default_rng(2)
    dims = [(61, 128), (128, 128), (128, 40)]
    w, b = _net(rng, dims)
    raw = rng.standard_normal((64, 61)).astype(np.float32)
    target = rng.uniform(0, 1, (64, 40))
    args = (raw, target, np.zeros(61, np.float32), np.ones(61, np.float32), w, b, 1.0 / 64)
    _, p1, dw1, _ = mlp_ref.forward_backward(*args, rounding=True)
    _, p0, dw0, _ = mlp_ref.forward_backward(*args, rounding=False)
    assert np.max(np.abs(p1 - p0)) < 2e-2
    for a, c in zip(dw1, dw0):
        assert np.linalg.norm(a - c) / np.linalg.norm(c) < 3e-2


def test_adam_matches_torch_optim():
    rng = np.random.default_rng(3)
    w0 = rng.standard_normal(50).astype(np.float32)
    grads = [rng.standard_normal(50).astype(np.float32) for _ in range(4)]
    p = torch.nn.Parameter(torch.tensor(w0))
    opt = torch.optim.Adam([p], lr=1e-3, betas=(0.9, 0.999), eps=1e-8)
    w, m, v = w0, np.zeros(50, np.float32), np.zeros(50, np.float32)
    for step, g in enumerate(grads, start=1):
        p.grad = torch.tensor(g)
        opt.step()
        w, m, v = mlp_ref.adam(w, m, v, g, step, 1e-3)
    np.testing.assert_allclose(w, p.detach().numpy(), rtol=0, atol=2e-7)
