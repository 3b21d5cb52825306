"""The CPU oracle reproduces the reference's own outputs (golden vectors).

Golden vectors were produced by running the reference (tests/golden/make_golden.py);
these tests pin oracle.restate to them so the oracle can check the GPU engine
on cases the golden set does not cover.
"""

import warnings

import numpy as np
import pytest

from conftest import SMALL_GOLDEN, golden_case, oracle_inputs
from oracle import restate


@pytest.mark.parametrize("name", SMALL_GOLDEN + ["co2_band_top3"])
def test_oracle_matches_reference_golden(name):
    sd, prof, prm, data = golden_case(name)
    nu = restate.grid(prm["nu_min"], prm["nu_max"], prm["step"])
    assert nu.size == int(data["n_nu"])
    inp = oracle_inputs(sd, prof)
    with warnings.catch_warnings(record=True) as wl:
        warnings.simplefilter("always")
        od = restate.optical_depth(nu, inp["lines"], inp["tips"], inp["masses"], inp["p_atm"],
                                   inp["t_layer"], inp["vmr_layer"], inp["col"], prm["cutoff"], prm["tile"])
    tau = od.sum(axis=0)
    np.testing.assert_allclose(tau, data["tau"], rtol=1e-13, atol=0)
    np.testing.assert_allclose(restate.transmittance(nu, od, prm["mu"]), data["T"], rtol=1e-12, atol=1e-300)
    if "od_layers" in data:
        np.testing.assert_allclose(od, data["od_layers"], rtol=1e-13, atol=0)
    got = sorted(str(w.message) for w in wl)
    want = sorted(m for m in data["warnings"].tolist() if m)
    assert got == want


def test_tile_width_changes_result_like_reference():
    """The reference's tile-window rule makes tau depend on tile_width (forward.py:295-301)."""
    _, _, _, d2 = golden_case("tile2.0")
    _, _, _, d05 = golden_case("tile0.5")
    rel = np.abs(d2["tau"] - d05["tau"]) / d2["tau"]
    assert rel.max() > 1e-2


def test_oracle_raises_on_negative_strength():
    sd, prof, prm, _ = golden_case("tile2.0")
    inp = oracle_inputs(sd, prof)
    inp["lines"] = dict(inp["lines"])
    inp["lines"]["Sref"] = inp["lines"]["Sref"].copy()
    inside = np.flatnonzero((inp["lines"]["nu0"] > 706.0) & (inp["lines"]["nu0"] < 711.0))
    inp["lines"]["Sref"][inside[3]] = -1e-22
    nu = restate.grid(prm["nu_min"], prm["nu_max"], prm["step"])
    with pytest.raises(FloatingPointError, match=r"Layer 0, gas 'CO2': non-finite or negative line strength"):
        restate.optical_depth(nu, inp["lines"], inp["tips"], inp["masses"], inp["p_atm"], inp["t_layer"],
                              inp["vmr_layer"], inp["col"], prm["cutoff"], prm["tile"])


def test_oracle_eval_count_small():
    sd, prof, prm, _ = golden_case("tile0.5")
    inp = oracle_inputs(sd, prof)
    nu = restate.grid(prm["nu_min"], prm["nu_max"], prm["step"])
    n = restate.count_evals(nu, inp["lines"], inp["tips"], inp["masses"], inp["p_atm"], inp["t_layer"],
                            inp["vmr_layer"], inp["col"], prm["cutoff"], prm["tile"])
    # brute force over layers x tiles x lines
    tile = max(1, int(np.floor(prm["tile"] / (nu[1] - nu[0]) + 1e-8)))
    brute = 0
    grp = restate.prepare_groups(nu, inp["lines"], inp["tips"], inp["masses"], tuple(inp["col"]),
                                 inp["p_atm"], inp["t_layer"], prm["cutoff"])
    for k in range(inp["p_atm"].size):
        for g in grp:
            lp = restate.line_params(k, inp["lines"], inp["p_atm"], inp["t_layer"], inp["vmr_layer"],
                                     inp["col"], g)
            if lp is None:
                continue
            shifted = lp[1]
            for t0 in range(0, nu.size, tile):
                t1 = min(t0 + tile, nu.size)
                m = (shifted >= nu[t0] - prm["cutoff"]) & (shifted <= nu[t1 - 1] + prm["cutoff"])
                brute += int(m.sum()) * (t1 - t0)
    assert n == brute > 0
