"""Host-side logic of the drop-in API (no GPU): validation, layers, groups, config, output."""

import os
import warnings

import numpy as np
import pytest

import pylblrtm_b200 as lbl
from conftest import golden_case, oracle_inputs
from oracle import restate
from pylblrtm_b200 import engine
from pylblrtm_b200.atmosphere import AtmosphericProfile
from pylblrtm_b200.config import ForwardResult, _write, load_config
from pylblrtm_b200.spectral_data import SpectralData


# ---- AtmosphericProfile (atmosphere.py:63-100) ---------------------------------

@pytest.mark.parametrize("p,t,vmr,msg", [
    ([1.0], [200.0], {}, "at least 2 levels"),
    ([1.0, -2.0], [200.0, 210.0], {}, "finite and positive"),
    ([5.0, 2.0], [200.0, 210.0], {}, "strictly increasing"),
    ([1.0, 2.0], [200.0], {}, "same length as pressure_hpa"),
    ([1.0, 2.0], [200.0, 0.0], {}, "temperature_k must be finite and positive"),
    ([1.0, 2.0], [200.0, 210.0], {"CO2": [1e-4]}, r"vmr\['CO2'\] must have the same length"),
    ([1.0, 2.0], [200.0, 210.0], {"CO2": [1e-4, 1.5]}, r"must be finite and in \[0, 1\]"),
])
def test_profile_validation(p, t, vmr, msg):
    with pytest.raises(ValueError, match=msg):
        AtmosphericProfile(p, t, vmr)


def test_build_layers_matches_oracle_bitwise():
    prof = lbl.us_standard_atmosphere()
    lay = prof.build_layers()
    p, t, v, c = restate.build_layers(prof.pressure_hpa, prof.temperature_k, prof.vmr)
    assert np.array_equal(lay.pressure_atm, p) and np.array_equal(lay.temperature_k, t)
    for g in prof.vmr:
        assert np.array_equal(lay.vmr[g], v[g]) and np.array_equal(lay.column_cm2[g], c[g])


def test_standard_profile_shapes_and_errors():
    prof = lbl.us_standard_atmosphere(["CO2", "H2O"], alt_max_km=20.0)
    assert prof.n_levels == 15 and prof.pressure_hpa[0] < prof.pressure_hpa[-1]
    assert lbl.list_profile_gases() == ["H2O", "CO2", "O3", "N2O", "CH4", "CO"]
    with pytest.raises(ValueError, match="Unknown gas"):
        lbl.us_standard_atmosphere(["XX"])
    with pytest.raises(ValueError, match="alt_max_km"):
        lbl.us_standard_atmosphere(alt_max_km=60.0)


# ---- SpectralData.Q (spectral_data.py:43-52; reference tests test_spectral_data.py:72-92) ----

def _sd():
    t = np.arange(100.0, 400.0, 10.0)
    lines = {k: np.zeros(3) for k in ("nu0", "Sref", "g_air", "g_self", "Elow", "n_air", "shift")}
    lines["nu0"] = np.array([700.0, 701.0, 702.0])
    lines["mol_id"] = np.array([1, 1, 1])
    lines["iso_id"] = np.array([1, 1, 2])
    return SpectralData(lines, {(1, 1): (t, t / 2.0), (1, 2): (t, t * 3.0)}, {(1, 1): 18.0})


def test_q_interpolation_and_clamp():
    sd = _sd()
    assert sd.Q(296.0, 1, 1) == pytest.approx(148.0)
    assert sd.Q(155.0, np.int64(1), np.int32(2)) == pytest.approx(465.0)
    assert sd.Q(50.0, 1, 1) == 50.0 and sd.Q(1e4, 1, 1) == 195.0
    with pytest.raises(KeyError, match=r"No TIPS data for \(mol_id=2, iso_id=1\)"):
        sd.Q(296.0, 2, 1)
    assert sd.n_lines == 3 and "2 lines" not in repr(sd) and "3 lines" in repr(sd)


# ---- grid and tile sizes (forward.py:141-142, 175-176) ----------------------------

@pytest.mark.parametrize("lo,hi,step,tw", [(700.0, 750.0, 0.001, 2.0), (600.0, 2500.0, 0.001, 2.0),
                                           (701.3, 758.9, 0.01, 2.0), (705.0, 712.0, 0.001, 0.5),
                                           (0.5, 3.7, 0.0007, 0.3)])
def test_grid_and_tile_match_reference_formula(lo, hi, step, tw):
    g = engine.make_grid(lo, hi, step, tw)
    nu = restate.grid(lo, hi, step)
    assert g.n_nu == nu.size and np.array_equal(g.nu, nu)
    assert g.tile_samples == max(1, int(np.floor(tw / (nu[1] - nu[0]) + 1e-8)))
    g2 = engine.grid_from_array(nu, tw)
    assert np.array_equal(g2.nu, nu) and g2.tile_samples == g.tile_samples


def test_grid_from_array_rejects_nonuniform():
    with pytest.raises(ValueError, match="uniform grid"):
        engine.grid_from_array(np.array([1.0, 2.0, 4.0]), 2.0)


# ---- group selection (forward.py:189-245) ----------------------------------------

def test_group_selection_matches_oracle_on_edge_case():
    sd, prof, prm, data = golden_case("edge_mix")
    inp = oracle_inputs(sd, prof)
    nu = restate.grid(prm["nu_min"], prm["nu_max"], prm["step"])
    with warnings.catch_warnings(record=True) as w1:
        warnings.simplefilter("always")
        ref = restate.prepare_groups(nu, inp["lines"], inp["tips"], inp["masses"], tuple(inp["col"]),
                                     inp["p_atm"], inp["t_layer"], prm["cutoff"])
    with warnings.catch_warnings(record=True) as w2:
        warnings.simplefilter("always")
        groups, gid = engine.select_groups(sd, list(prof.vmr), nu[0], nu[-1], prm["cutoff"],
                                           float(inp["p_atm"].max()), 2)
    assert [(g.mol_id, g.iso_id, g.gas, g.molar_mass) for g in groups] == \
        [(m, i, gas, mm) for m, i, gas, _, mm, _ in ref]
    assert sorted(str(w.message) for w in w1) == sorted(str(w.message) for w in w2)
    for gi, (m, i, _, _, _, _) in enumerate(ref):
        sel = (sd.lines["mol_id"] == m) & (sd.lines["iso_id"] == i)
        assert np.all(gid[sel] == gi)
    assert np.all(gid[~np.isin(gid, range(len(groups)))] == -1)


def test_group_selection_missing_tips_raises_keyerror():
    sd, prof, prm, _ = golden_case("tile2.0")
    sd2 = SpectralData(sd.lines, {}, sd.molar_masses, sd.molecule)
    with pytest.raises(KeyError, match=r"No TIPS data for \(mol_id=2, iso_id=1\)"):
        engine.select_groups(sd2, list(prof.vmr), 705.0, 712.0, 1.0, 1.0, 2)


def test_group_selection_large_ids_use_unique_path():
    sd = _sd()
    sd.lines["mol_id"] = np.array([1, 1, 5000])
    with warnings.catch_warnings(record=True) as wl:
        warnings.simplefilter("always")
        groups, gid = engine.select_groups(sd, ["H2O"], 699.0, 703.0, 5.0, 1.0, 2)
    assert [(g.mol_id, g.iso_id) for g in groups] == [(1, 1)]
    assert gid.tolist() == [0, 0, -1]
    msgs = [str(w.message) for w in wl]
    assert any("mol_id=5000 is not in the HITRAN catalogue" in m for m in msgs)


# ---- config (config.py:23-124) and output (config.py:129-319) ----------------------

def test_load_config_defaults_and_merge(tmp_path):
    cfg = load_config({"spectral": {"nu_min_cm1": 710}})
    assert cfg["spectral"]["nu_min_cm1"] == 710 and cfg["spectral"]["nu_max_cm1"] == 750.0
    assert cfg["output"]["save"]["format"] == "npz"
    y = tmp_path / "c.yaml"
    y.write_text("spectral:\n  step_cm1: 0.01\noutput:\n  optical_depth: true\n")
    cfg = load_config(str(y))
    assert cfg["spectral"]["step_cm1"] == 0.01 and cfg["output"]["optical_depth"] is True
    with pytest.raises(FileNotFoundError):
        load_config(str(tmp_path / "missing.yaml"))


@pytest.mark.parametrize("over,msg", [
    ({"spectral": {"nu_min_cm1": 800}}, "nu_min_cm1 must be strictly less"),
    ({"spectral": {"step_cm1": 0}}, "step_cm1 must be positive"),
    ({"calculation": {"line_cutoff_cm1": 0}}, "line_cutoff_cm1 must be positive"),
    ({"calculation": {"mu_view": 1.5}}, "mu_view must be in"),
    ({"output": {"transmittance": False}}, "At least one output"),
    ({"output": {"save": {"format": "xls"}}}, "format must be"),
    ({"engine": {"precision": "fp16"}}, "engine.precision"),
])
def test_config_validation(over, msg):
    with pytest.raises(ValueError, match=msg):
        load_config(over)


def test_forward_result_save_formats(tmp_path, capsys):
    nu = np.linspace(700, 701, 5)
    r = ForwardResult(nu, load_config({}), transmittance=np.full(5, 0.5), optical_depth=np.ones(5),
                      optical_depth_layers=np.ones((2, 5)))
    p = r.save(path=str(tmp_path), fmt="npz", prefix="a")
    d = np.load(p)
    assert set(d.files) == {"wavenumber_cm1", "transmittance", "optical_depth", "optical_depth_layers"}
    p = _write(r, str(tmp_path), "csv", "b")
    lines = open(p).read().splitlines()
    assert lines[0] == "wavenumber_cm1,transmittance,optical_depth" and len(lines) == 6
    p = _write(r, str(tmp_path), "txt", "c")
    assert open(p).read().splitlines()[0] == "wavenumber_cm1\ttransmittance\toptical_depth"
    assert "Saved:" in capsys.readouterr().out
    assert "optical_depth_layers[2, 5]" in repr(r)


def test_api_type_and_range_errors():
    sd = _sd()
    prof = lbl.us_standard_atmosphere(["H2O"])
    with pytest.raises(TypeError):
        lbl.compute_transmittance(None, prof, 700, 701)
    with pytest.raises(TypeError):
        lbl.compute_transmittance(sd, None, 700, 701)
    with pytest.raises(ValueError, match="strictly less"):
        lbl.compute_transmittance(sd, prof, 701, 700)
    with pytest.raises(ValueError, match="step_cm1"):
        lbl.compute_transmittance(sd, prof, 700, 701, step_cm1=0)
    with pytest.raises(ValueError, match="mu_view"):
        lbl.compute_transmittance(sd, prof, 700, 701, mu_view=0)
    with pytest.raises(TypeError):
        lbl.run_forward(sd, None, {})


def test_batch_validation_errors():
    sd = _sd()
    p = np.array([[1.0, 10.0, 100.0], [1.0, 10.0, 100.0]])
    t = np.full_like(p, 250.0)
    with pytest.raises(ValueError, match="strictly increasing"):
        lbl.transmittance_batch(sd, p[:, ::-1], t, {"H2O": np.full_like(p, 1e-3)}, 700, 701)
    with pytest.raises(ValueError, match=r"vmr\['H2O'\] must be finite and in \[0, 1\]"):
        lbl.transmittance_batch(sd, p, t, {"H2O": np.full_like(p, 2.0)}, 700, 701)
    with pytest.raises(ValueError, match="mu_view"):
        lbl.transmittance_batch(sd, p, t, {"H2O": np.full_like(p, 1e-3)}, 700, 701, mu_view=[1.0, 0.0])
    with pytest.raises(TypeError):
        lbl.transmittance_batch(None, p, t, {}, 700, 701)
