"""Layer Jacobians of the float32 engine (lbl_jacobian_ml_f32) and the autograd wrapper.

Checked against (1) the engine's float64 optical depth, (2) autograd of the float64
torch restatement (oracle/torch_ref.py) and (3) central finite differences
(dT = 1e-3 K, d ln VMR = 1e-3) of the float64 oracle on 8 seeded perturbed 60-layer
profiles. Tolerance for the float32 Jacobian: 2e-4 of the largest |derivative| of
the layer, elementwise. The d/dlnVMR differences use only the H2O lines (the other
gases' lines do not depend on the H2O mixing ratio), so the difference is not lost
in the rounding of the other gases' optical depth.
"""

import numpy as np
import pytest
import torch

from oracle import restate, torch_ref
from pylblrtm_b200 import adjoint, engine, synthetic
from pylblrtm_b200.atmosphere import COLUMN_FACTOR
from pylblrtm_b200.spectral_data import SpectralData

pytestmark = pytest.mark.gpu

JAC_TOL = 2e-4


def _small():
    sd = synthetic.restrict(synthetic.three_gas_lines(6000, 1492, 1512, seed=3), 1492, 1512)
    prof = synthetic.profile_from_levels(synthetic.logp_levels(6))
    return sd, prof


def _only(sd, mol):
    keep = sd.lines["mol_id"] == mol
    return SpectralData({k: v[keep] for k, v in sd.lines.items()}, sd.tips, sd.molar_masses)


def test_jacobian_od_matches_forward(cuda):
    sd, prof = _small()
    j = adjoint.layer_jacobians(sd, prof, 1499.0, 1503.0, step_cm1=0.001)
    res = engine.optical_depth(sd, engine.layer_input_from_profile(prof),
                               engine.make_grid(1499.0, 1503.0, 0.001, 2.0), 25.0, precision="fp64", want_od=True)
    od64 = res.od[0].cpu().numpy()
    assert np.max(np.abs(j["od"] - od64) / od64) < 2e-5


def test_jacobian_against_torch_autograd(cuda):
    sd, prof = _small()
    nu = restate.grid(1500.0, 1500.6, 0.003)
    j = adjoint.layer_jacobians(sd, prof, 1500.0, 1500.6, step_cm1=0.003)
    p, t, v, c = restate.build_layers(prof.pressure_hpa, prof.temperature_k, prof.vmr)
    air = COLUMN_FACTOR * (np.abs(np.diff(prof.pressure_hpa)) * 100.0) / 1e4
    rng = np.random.default_rng(2)
    for k in range(p.size):
        tt = torch.tensor(t, requires_grad=True)
        lv = torch.tensor(np.log(v["H2O"]), requires_grad=True)
        vm = {g: (torch.exp(lv) if g == "H2O" else torch.tensor(v[g])) for g in v}
        odk = torch_ref.layer_optical_depth(nu, sd.lines, sd.tips, sd.molar_masses, p, tt, vm, air, k)
        w = rng.normal(size=nu.size)
        (odk * torch.tensor(w)).sum().backward()
        got_t = float((j["dtau_dT"][k] * w).sum())
        got_v = float((j["dtau_dlnvmr"][k] * w).sum())
        scale_t = np.abs(j["dtau_dT"][k]).sum()
        scale_v = np.abs(j["dtau_dlnvmr"][k]).sum()
        assert abs(got_t - tt.grad[k].item()) <= JAC_TOL * scale_t, (k, got_t, tt.grad[k].item())
        assert abs(got_v - lv.grad[k].item()) <= JAC_TOL * scale_v, (k, got_v, lv.grad[k].item())


@pytest.mark.parametrize("seed", range(8))
def test_jacobian_against_central_differences(cuda, seed):
    """8 seeded perturbed 60-layer profiles, 1000-1200 cm^-1 lines, 0.5 cm^-1 window, 5 layers each."""
    lines = synthetic.restrict(synthetic.three_gas_lines(), 1000.0, 1200.0)
    lo, hi = 1100.0, 1100.5
    sd = synthetic.restrict(lines, lo - 26.0, hi + 26.0)
    sd_h2o = _only(sd, 1)
    lv_all = synthetic.perturbed_levels(synthetic.logp_levels(), 8, seed=2024)
    prof = synthetic.profile_from_levels(lv_all, seed)
    j = adjoint.layer_jacobians(sd, prof, lo, hi)
    nu = j["nu"]
    p, t, v, c = restate.build_layers(prof.pressure_hpa, prof.temperature_k, prof.vmr)
    air = COLUMN_FACTOR * (np.abs(np.diff(prof.pressure_hpa)) * 100.0) / 1e4

    def od_k(data, k, dt=0.0, dlnv=0.0):
        sl = slice(k, k + 1)
        v2 = {g: a[sl].copy() for g, a in v.items()}
        c2 = {g: a[sl].copy() for g, a in c.items()}
        v2["H2O"] = v2["H2O"] * np.exp(dlnv)
        c2["H2O"] = v2["H2O"] * air[sl]
        return restate.optical_depth(nu, data.lines, data.tips, data.molar_masses, p[sl], t[sl] + dt, v2, c2)[0]

    h = 1e-3
    for k in (5, 20, 35, 50, 59):
        fd_t = (od_k(sd, k, dt=h) - od_k(sd, k, dt=-h)) / (2 * h)
        fd_v = (od_k(sd_h2o, k, dlnv=h) - od_k(sd_h2o, k, dlnv=-h)) / (2 * h)
        assert np.max(np.abs(j["dtau_dT"][k] - fd_t)) <= JAC_TOL * np.max(np.abs(fd_t)), k
        assert np.max(np.abs(j["dtau_dlnvmr"][k] - fd_v)) <= JAC_TOL * np.max(np.abs(fd_v)), k


def test_autograd_function_backward_matches_jacobian(cuda):
    sd, prof = _small()
    profs = [prof, synthetic.profile_from_levels(synthetic.perturbed_levels(synthetic.logp_levels(6), 1, 9), 0)]
    state = adjoint.LayerState.from_profiles(sd, profs, "H2O", 1499.0, 1502.0)
    t_layer = torch.tensor(np.stack([p.build_layers().temperature_k for p in profs]), device=cuda,
                           requires_grad=True)
    lnv = torch.tensor(np.log(state.vmr["H2O"]), device=cuda, requires_grad=True)
    tau = adjoint.layer_optical_depth(t_layer, lnv, state)
    assert tau.shape == (2, state.grid.n_nu) and tau.dtype == torch.float64
    w = torch.randn(tau.shape, dtype=torch.float64, device=cuda)
    (tau * w).sum().backward()
    for b, prof_b in enumerate(profs):
        j = adjoint.layer_jacobians(sd, prof_b, 1499.0, 1502.0)
        wb = w[b].cpu().numpy()
        ref_t = (j["dtau_dT"] * wb).sum(axis=1)
        ref_v = (j["dtau_dlnvmr"] * wb).sum(axis=1)
        np.testing.assert_allclose(t_layer.grad[b].cpu().numpy(), ref_t, rtol=1e-5,
                                   atol=1e-6 * np.abs(ref_t).max())
        np.testing.assert_allclose(lnv.grad[b].cpu().numpy(), ref_v, rtol=1e-5,
                                   atol=1e-6 * np.abs(ref_v).max())


def test_batched_jacobians_match_single_profiles_and_stream(cuda):
    from pylblrtm_b200 import batch
    sd, _ = _small()
    lv = synthetic.perturbed_levels(synthetic.logp_levels(6), 3, seed=77)
    vmr = {g: lv[g] for g in ("H2O", "CO2", "O3")}
    lo, hi = 1500.0, 1503.0
    mu = np.array([1.0, 0.7, 0.55])
    res = adjoint.layer_jacobians_batch(sd, lv["p"], lv["t"], vmr, lo, hi, mu_view=mu, profiles_per_launch=2,
                                        deterministic=True)
    for i in range(3):
        one = adjoint.layer_jacobians(sd, synthetic.profile_from_levels(lv, i), lo, hi, as_numpy=False,
                                      deterministic=True)
        for k in ("od", "dtau_dT", "dtau_dlnvmr"):
            assert torch.equal(res[k][i], one[k]), (i, k)
    chunks = []
    out = adjoint.layer_jacobians_batch(sd, lv["p"], lv["t"], vmr, lo, hi, mu_view=mu, profiles_per_launch=2,
                                        on_chunk=lambda sl, o: chunks.append((sl, {k: v.clone() for k, v in o.items()})),
                                        deterministic=True)
    assert out is None and [c[0] for c in chunks] == [slice(0, 2), slice(2, 3)]
    for k in ("od", "dtau_dT", "dtau_dlnvmr", "trans"):
        assert torch.equal(torch.cat([c[1][k] for c in chunks]), res[k])
    _, t_fwd = batch.transmittance_batch(sd, lv["p"], lv["t"], vmr, lo, hi, mu_view=mu, as_numpy=False)
    assert torch.max(torch.abs(res["trans"] - t_fwd)).item() <= 1e-5
    # the default (atomic) near-zone sums agree with the ordered ones to rounding
    fast = adjoint.layer_jacobians_batch(sd, lv["p"], lv["t"], vmr, lo, hi, mu_view=mu, profiles_per_launch=2)
    for k in ("od", "dtau_dT", "dtau_dlnvmr"):
        assert torch.max(torch.abs(fast[k] - res[k])).item() <= 1e-6 * torch.max(torch.abs(res[k])).item(), k
    with pytest.raises(ValueError, match="not in vmr"):
        adjoint.layer_jacobians_batch(sd, lv["p"], lv["t"], vmr, lo, hi, gas="CH4")
    with pytest.raises(ValueError, match="mu_view"):
        adjoint.layer_jacobians_batch(sd, lv["p"], lv["t"], vmr, lo, hi, mu_view=1.5)


@pytest.mark.parametrize("tile", [2.0, 5.0, 0.05, 0.3])
def test_jacobian_ranges_select_every_line(cuda, tile, monkeypatch):
    """Jacobians computed with the inner-line and near level-1 ranges equal, to float
    rounding, those of a scan of every candidate line (inner = near = NULL), with pressure
    shifts 40x the synthetic ones; tiles of one chunk, several chunks and below level 1's
    minimum size. A line lost by a range would change whole line profiles. The two scans
    group lines into different rounds, so the float sums run in another order, and the
    d/dT sums add terms of both signs: the bound is a few float roundings of the layer's
    largest value."""
    from pylblrtm_b200 import _lib
    sd = synthetic.restrict(synthetic.three_gas_lines(20000, 1490.0, 1520.0, seed=4), 1490.0, 1520.0)
    lines = {k: v.copy() for k, v in sd.lines.items()}
    lines["shift"] = lines["shift"] * 40.0
    sd = SpectralData(lines, dict(sd.tips), dict(sd.molar_masses), sd.molecule)
    lv = synthetic.perturbed_levels(synthetic.logp_levels(7), 2, seed=8)
    gases = ["H2O", "CO2", "O3"]
    li = engine.LayerInput(gases=gases, levels_p=lv["p"], levels_t=lv["t"],
                           levels_vmr=np.stack([lv[g] for g in gases], axis=1))
    job = engine.Job(sd, li, engine.make_grid(1500.0, 1510.3, 0.001, tile), 5.0)
    with_ranges = job.jacobian("H2O", deterministic=True)
    real_call = _lib.call

    def scan_all(name, *args):
        if name == "lbl_jacobian_ml_f32":
            args = args[:4] + (0, 0) + args[6:]
        return real_call(name, *args)

    monkeypatch.setattr(_lib, "call", scan_all)
    every = job.jacobian("H2O", deterministic=True)
    for a, b in zip(with_ranges, every):
        scale = b.abs().amax(dim=-1, keepdim=True).clamp_min(1e-30)
        assert ((a - b).abs() / scale).max().item() <= 5e-6
