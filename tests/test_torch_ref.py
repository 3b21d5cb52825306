"""The float64 torch restatement (oracle/torch_ref.py) against the oracle and finite differences.

It is the independent autograd reference for the engine's Jacobian kernel, so it is
pinned here: its optical depth equals oracle.restate (itself pinned to the
reference's golden vectors) and its gradients equal central differences of the
oracle.
"""

import numpy as np
import torch

from oracle import restate, torch_ref
from pylblrtm_b200 import synthetic
from pylblrtm_b200.atmosphere import COLUMN_FACTOR


def _case():
    sd = synthetic.restrict(synthetic.three_gas_lines(6000, 1492, 1512, seed=3), 1492, 1512)
    prof = synthetic.profile_from_levels(synthetic.logp_levels(6))
    p, t, v, c = restate.build_layers(prof.pressure_hpa, prof.temperature_k, prof.vmr)
    air = COLUMN_FACTOR * (np.abs(np.diff(prof.pressure_hpa)) * 100.0) / 1e4
    nu = restate.grid(1500.0, 1500.6, 0.003)
    return sd, p, t, v, c, air, nu


def test_weideman_matches_wofz():
    from scipy.special import wofz
    rng = np.random.default_rng(0)
    z = rng.uniform(-50, 50, 5000) + 1j * 10 ** rng.uniform(-4, 2, 5000)
    w = torch_ref.faddeeva(torch.tensor(z)).numpy()
    assert np.max(np.abs(w - wofz(z)) / np.abs(wofz(z))) < 1e-12


def test_torch_forward_and_gradients():
    sd, p, t, v, c, air, nu = _case()
    od = restate.optical_depth(nu, sd.lines, sd.tips, sd.molar_masses, p, t, v, c, 25.0, 2.0)
    k = 3
    tt = torch.tensor(t, requires_grad=True)
    lv = torch.tensor(np.log(v["H2O"]), requires_grad=True)
    vm = {g: (torch.exp(lv) if g == "H2O" else torch.tensor(v[g])) for g in v}
    odk = torch_ref.layer_optical_depth(nu, sd.lines, sd.tips, sd.molar_masses, p, tt, vm, air, k)
    np.testing.assert_allclose(odk.detach().numpy(), od[k], rtol=1e-12)
    w = torch.tensor(np.random.default_rng(1).normal(size=nu.size))
    (odk * w).sum().backward()

    def od_k(tk=None, lnv=None):
        t2 = t.copy()
        v2 = {g: a.copy() for g, a in v.items()}
        c2 = {g: a.copy() for g, a in c.items()}
        if tk is not None:
            t2[k] = tk
        if lnv is not None:
            v2["H2O"][k] = np.exp(lnv)
            c2["H2O"][k] = v2["H2O"][k] * air[k]
        sl = slice(k, k + 1)
        return restate.optical_depth(nu, sd.lines, sd.tips, sd.molar_masses, p[sl], t2[sl],
                                     {g: a[sl] for g, a in v2.items()}, {g: a[sl] for g, a in c2.items()})[0]
    h = 1e-3
    fd_t = ((od_k(tk=t[k] + h) - od_k(tk=t[k] - h)) / (2 * h) * w.numpy()).sum()
    lv0 = np.log(v["H2O"][k])
    fd_v = ((od_k(lnv=lv0 + h) - od_k(lnv=lv0 - h)) / (2 * h) * w.numpy()).sum()
    assert abs(tt.grad[k].item() - fd_t) <= 1e-7 * abs(fd_t)
    assert abs(lv.grad[k].item() - fd_v) <= 1e-5 * abs(fd_v)
