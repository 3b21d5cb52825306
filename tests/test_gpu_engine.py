"""GPU engine parity: device kernels against the reference's golden vectors and the oracle.

Tolerances (stated per the spec): float64 engine |dT| <= 1e-6, float32 engine
|dT| <= 1e-5; relative optical-depth errors are bounded separately because
several goldens are optically thick (T ~ 0 everywhere makes |dT| vacuous).
"""

import warnings

import numpy as np
import pytest
import torch

import pylblrtm_b200 as lbl
from conftest import ALL_GOLDEN, SMALL_GOLDEN, golden_case, oracle_inputs
from oracle import restate
from pylblrtm_b200 import _lib, engine, synthetic
from pylblrtm_b200.atmosphere import COLUMN_FACTOR
from pylblrtm_b200.spectral_data import SpectralData

pytestmark = pytest.mark.gpu

TOL = {"fp64": dict(dT=1e-6, rtau=1e-9, rod=1e-9), "fp32": dict(dT=1e-5, rtau=2e-5, rod=3e-5),
       "fp32-direct": dict(dT=1e-5, rtau=2e-5, rod=3e-5)}


def _run(sd, prof, prm, precision, layers=False, deterministic=False):
    cfg = {"spectral": {"nu_min_cm1": prm["nu_min"], "nu_max_cm1": prm["nu_max"], "step_cm1": prm["step"]},
           "calculation": {"mu_view": prm["mu"], "line_cutoff_cm1": prm["cutoff"],
                           "tile_width_cm1": prm["tile"]},
           "output": {"transmittance": True, "optical_depth": True, "optical_depth_layers": layers},
           "engine": {"precision": precision, "deterministic": deterministic}}
    with warnings.catch_warnings(record=True) as wl:
        warnings.simplefilter("always")
        res = lbl.run_forward(sd, prof, cfg)
    return res, sorted(str(w.message) for w in wl)


def _rel(a, b):
    den = np.abs(b)
    m = den > 1e-300
    return float(np.max(np.abs(a - b)[m] / den[m])) if m.any() else 0.0


@pytest.mark.parametrize("precision", ["fp64", "fp32", "fp32-direct"])
@pytest.mark.parametrize("name", ALL_GOLDEN)
def test_golden(cuda, name, precision):
    sd, prof, prm, data = golden_case(name)
    res, warns = _run(sd, prof, prm, precision, layers="od_layers" in data)
    tol = TOL[precision]
    assert res.wavenumber_cm1.size == int(data["n_nu"])
    assert np.max(np.abs(res.transmittance - data["T"])) <= tol["dT"]
    assert _rel(res.optical_depth, data["tau"]) <= tol["rtau"]
    if "od_layers" in data:
        assert _rel(res.optical_depth_layers, data["od_layers"]) <= tol["rod"]
    assert warns == sorted(m for m in data["warnings"].tolist() if m)


def test_compute_transmittance_matches_golden(cuda):
    sd, prof, prm, data = golden_case("tile0.5")
    nu, T = lbl.compute_transmittance(sd, prof, prm["nu_min"], prm["nu_max"], step_cm1=prm["step"],
                                      line_cutoff_cm1=prm["cutoff"], tile_width_cm1=prm["tile"],
                                      mu_view=prm["mu"], precision="fp64")
    assert nu.dtype == np.float64 and T.dtype == np.float64
    assert np.array_equal(nu, restate.grid(prm["nu_min"], prm["nu_max"], prm["step"]))
    assert np.max(np.abs(T - data["T"])) <= 1e-9


def test_internal_build_optical_depth(cuda):
    from pylblrtm_b200.forward import _build_optical_depth
    sd, prof, prm, data = golden_case("tile2.0")
    nu = restate.grid(prm["nu_min"], prm["nu_max"], prm["step"])
    od = _build_optical_depth(nu, sd, prof.build_layers(), prm["cutoff"], prm["tile"], precision="fp64")
    assert od.shape == data["od_layers"].shape and od.dtype == np.float64
    assert _rel(od, data["od_layers"]) <= 1e-9


def test_layers_built_on_device_bitwise(cuda):
    import torch
    for prof in (lbl.us_standard_atmosphere(), synthetic.logp_profile()):
        li = engine.layer_input_from_profile(prof)
        n_gas, n_lev = len(li.gases), prof.n_levels
        p = torch.tensor(li.levels_p, device=cuda)
        t = torch.tensor(li.levels_t, device=cuda)
        v = torch.tensor(li.levels_vmr, device=cuda)
        outs = [torch.empty((1, n_lev - 1), dtype=torch.float64, device=cuda) for _ in range(2)]
        vo = [torch.empty((1, n_gas, n_lev - 1), dtype=torch.float64, device=cuda) for _ in range(2)]
        _lib.call("lbl_build_layers", p.data_ptr(), t.data_ptr(), v.data_ptr(), 1, n_lev, n_gas, COLUMN_FACTOR,
                  outs[0].data_ptr(), outs[1].data_ptr(), vo[0].data_ptr(), vo[1].data_ptr(),
                  torch.cuda.current_stream().cuda_stream)
        host = prof.build_layers()
        assert np.array_equal(outs[0].cpu().numpy()[0], host.pressure_atm)
        assert np.array_equal(outs[1].cpu().numpy()[0], host.temperature_k)
        for gi, g in enumerate(li.gases):
            assert np.array_equal(vo[0].cpu().numpy()[0, gi], host.vmr[g])
            assert np.array_equal(vo[1].cpu().numpy()[0, gi], host.column_cm2[g])


def test_partition_ratio_on_device_matches_np_interp(cuda):
    import torch
    prof = synthetic.logp_profile()
    host = prof.build_layers()
    tables = [synthetic.tips_power_law(174.0), synthetic.tips_power_law(3483.0, 150.0, 400.0, 2.5),
              (np.array([200.0, 230.0, 250.0]), np.array([100.0, 150.0, 120.0]))]   # clamps both ends
    gases = list(prof.vmr)
    n_lay, n_grp = host.n_layers, len(tables)
    f = lambda a, dt=torch.float64: torch.tensor(np.asarray(a), dtype=dt, device=cuda)
    t_l, p_l = f(host.temperature_k), f(host.pressure_atm)
    v_l = f(np.stack([host.vmr[g] for g in gases]))
    c_l = f(np.stack([host.column_cm2[g] for g in gases]))
    offs = np.cumsum([0] + [t.size for t, _ in tables[:-1]])
    out = torch.empty(n_lay * n_grp * 6, dtype=torch.float64, device=cuda)
    # every argument tensor stays referenced until the kernel has run
    args = [f([0, 1, 2], torch.int32), f([18.01, 47.98, 43.99]), f(offs, torch.int32),
            f([t.size for t, _ in tables], torch.int32), f(np.concatenate([t for t, _ in tables])),
            f(np.concatenate([q for _, q in tables]))]
    _lib.call("lbl_layer_groups", t_l.data_ptr(), p_l.data_ptr(), v_l.data_ptr(), c_l.data_ptr(), 1, n_lay,
              len(gases), n_grp, *[a.data_ptr() for a in args], out.data_ptr(),
              torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    lg = out.cpu().numpy().reshape(n_lay, n_grp, 6)
    for g, (tt, qq) in enumerate(tables):
        gas = gases[g]
        for k in range(n_lay):
            T, P = host.temperature_k[k], host.pressure_atm[k]
            assert lg[k, g, 4] == np.interp(296.0, tt, qq) / np.interp(float(T), tt, qq)
            p_self = host.vmr[gas][k] * P
            assert lg[k, g, 1] == p_self and lg[k, g, 2] == P - p_self
            assert lg[k, g, 3] == host.column_cm2[gas][k]


def test_eval_count_matches_oracle(cuda):
    sd, prof, prm, _ = golden_case("edge_mix")
    grid = engine.make_grid(prm["nu_min"], prm["nu_max"], prm["step"], prm["tile"])
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        res = engine.optical_depth(sd, engine.layer_input_from_profile(prof), grid, prm["cutoff"],
                                   precision="fp32", count_evals=True)
        inp = oracle_inputs(sd, prof)
        n = restate.count_evals(grid.nu, inp["lines"], inp["tips"], inp["masses"], inp["p_atm"],
                                inp["t_layer"], inp["vmr_layer"], inp["col"], prm["cutoff"], prm["tile"])
    assert res.evals == n > 0


@pytest.mark.parametrize("precision", ["fp64", "fp32", "fp32-direct"])
def test_nonfinite_or_negative_strength_raises(cuda, precision):
    sd, prof, prm, _ = golden_case("edge_mix")
    lines = {k: v.copy() for k, v in sd.lines.items()}
    co2 = np.flatnonzero((lines["mol_id"] == 2) & (lines["iso_id"] == 1) & (lines["nu0"] > 700.5))
    lines["Sref"][co2[0]] = np.nan
    bad = SpectralData(lines, sd.tips, sd.molar_masses)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        with pytest.raises(FloatingPointError, match=r"^Layer 0, gas 'CO2': non-finite or negative line strength$"):
            lbl.compute_transmittance(bad, prof, prm["nu_min"], prm["nu_max"], step_cm1=prm["step"],
                                      line_cutoff_cm1=prm["cutoff"], tile_width_cm1=prm["tile"],
                                      precision=precision)


def test_deferred_error_check_raises_later(cuda):
    """Job.run(defer_errors=True) queues every stage and returns; result.check() then raises
    the same error the blocking call raises, and a clean run's check() passes."""
    sd, prof, prm, _ = golden_case("edge_mix")
    lines = {k: v.copy() for k, v in sd.lines.items()}
    co2 = np.flatnonzero((lines["mol_id"] == 2) & (lines["iso_id"] == 1) & (lines["nu0"] > 700.5))
    lines["Sref"][co2[0]] = np.nan
    grid = engine.make_grid(prm["nu_min"], prm["nu_max"], prm["step"], prm["tile"])
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        good = engine.Job(sd, engine.layer_input_from_profile(prof), grid, prm["cutoff"])
        bad = engine.Job(SpectralData(lines, sd.tips, sd.molar_masses), engine.layer_input_from_profile(prof), grid,
                         prm["cutoff"])
    rb = bad.run("fp32", mu=[1.0], want_od=False, want_trans=True, defer_errors=True)
    rg = good.run("fp32", mu=[1.0], want_od=False, want_trans=True, defer_errors=True)
    rg.check()
    with pytest.raises(FloatingPointError, match=r"^Layer 0, gas 'CO2': non-finite or negative line strength$"):
        rb.check()
    rb.check()                                      # raised once; the check is then spent
    ref = good.run("fp32", mu=[1.0], want_od=False, want_trans=True)
    assert torch.allclose(rg.trans, ref.trans, rtol=1e-6, atol=0)


def test_missing_tips_raises_keyerror(cuda):
    sd, prof, prm, _ = golden_case("tile2.0")
    with pytest.raises(KeyError, match="No TIPS data"):
        lbl.compute_transmittance(SpectralData(sd.lines, {}, sd.molar_masses), prof, 705.0, 712.0)


def test_no_contributing_lines_gives_unit_transmittance(cuda):
    sd = synthetic.co2_band(100, 900.0, 950.0)
    nu, T = lbl.compute_transmittance(sd, lbl.us_standard_atmosphere(["CO2"]), 700.0, 710.0, step_cm1=0.01)
    assert np.all(T == 1.0) and nu.size == 1001


def test_fp32_is_deterministic(cuda):
    sd, prof, prm, _ = golden_case("coarse_step")
    a = _run(sd, prof, prm, "fp32", layers=True, deterministic=True)[0]
    b = _run(sd, prof, prm, "fp32", layers=True, deterministic=True)[0]
    assert np.array_equal(a.optical_depth_layers, b.optical_depth_layers)


@pytest.mark.parametrize("seed", [1, 2, 3, 4])
def test_random_cases_against_oracle(cuda, seed):
    """Seeded small cases with mixed groups, odd tiles, grids and cutoffs against the oracle."""
    rng = np.random.default_rng(seed)
    lo = float(rng.uniform(600, 2400))
    width = float(rng.uniform(1, 6))
    step = float(rng.choice([0.001, 0.0025, 0.004]))
    cutoff = float(rng.uniform(0.5, 8))
    tile = float(rng.uniform(0.2, 3))
    sd = synthetic.restrict(synthetic.three_gas_lines(20000, lo - cutoff - 1, lo + width + cutoff + 1,
                                                      seed=seed), lo - cutoff - 1, lo + width + cutoff + 1)
    lv = synthetic.logp_levels(int(rng.integers(3, 12)))
    prof = synthetic.profile_from_levels(lv)
    mu = float(rng.uniform(0.3, 1.0))
    prm = dict(nu_min=lo, nu_max=lo + width, step=step, cutoff=cutoff, tile=tile, mu=mu)
    inp = oracle_inputs(sd, prof)
    nu = restate.grid(lo, lo + width, step)
    od = restate.optical_depth(nu, inp["lines"], inp["tips"], inp["masses"], inp["p_atm"], inp["t_layer"],
                               inp["vmr_layer"], inp["col"], cutoff, tile)
    tau, T = od.sum(0), restate.transmittance(nu, od, mu)
    for precision in ("fp64", "fp32", "fp32-direct"):
        res, _ = _run(sd, prof, prm, precision, layers=True)
        tol = TOL[precision]
        assert np.max(np.abs(res.transmittance - T)) <= tol["dT"]
        assert _rel(res.optical_depth, tau) <= tol["rtau"]
        assert _rel(res.optical_depth_layers, od) <= tol["rod"]


def test_full_size_three_gas_fp32_against_fp64(cuda):
    """200k lines x 60 layers x 1.9M points: size-independent agreement of the engines."""
    sd = synthetic.three_gas_lines()
    prof = synthetic.logp_profile()
    grid = engine.make_grid(600.0, 2500.0, 0.001, 2.0)
    li = engine.layer_input_from_profile(prof)
    r = {p: engine.optical_depth(sd, li, grid, 25.0, precision=p, mu=[0.8], want_od=True, want_tau=True,
                                 want_trans=True, count_evals=True) for p in ("fp64", "fp32", "fp32-direct")}
    assert r["fp32"].evals == r["fp32-direct"].evals == r["fp64"].evals > 6e11
    assert r["fp32"].work < r["fp32"].evals / 20          # the multi-level split does far fewer evaluations
    t64 = r["fp64"].tau[0].cpu().numpy()
    od64 = r["fp64"].od[0]
    assert np.all(t64 > 0)
    for p in ("fp32", "fp32-direct"):
        assert _rel(r[p].tau[0].cpu().numpy(), t64) <= 2e-5
        assert np.max(np.abs(r[p].trans[0].cpu().numpy() - r["fp64"].trans[0].cpu().numpy())) <= 1e-5
        rel_od = ((r[p].od[0].double() - od64).abs() / od64.abs()).max().item()
        assert rel_od <= 3e-5, (p, rel_od)


def test_batch_equals_single_profiles_bitwise(cuda):
    """A batch of perturbed profiles gives exactly the per-profile spectra."""
    sd = synthetic.restrict(synthetic.three_gas_lines(30000, 1480.0, 1540.0, seed=9), 1480.0, 1540.0)
    lv = synthetic.perturbed_levels(synthetic.logp_levels(13), 3, seed=5)
    mu = np.array([1.0, 0.7, 0.45])
    for precision in ("fp32", "fp64"):
        nu, tb = lbl.transmittance_batch(sd, lv["p"], lv["t"], {g: lv[g] for g in ("H2O", "CO2", "O3")},
                                         1500.0, 1510.0, mu_view=mu, precision=precision, deterministic=True)
        for i in range(3):
            _, t1 = lbl.compute_transmittance(sd, synthetic.profile_from_levels(lv, i), 1500.0, 1510.0,
                                              mu_view=float(mu[i]), precision=precision, deterministic=True)
            assert np.array_equal(tb[i], t1), (precision, i)


def test_channel_mean_matches_host_box_average(cuda):
    sd = synthetic.restrict(synthetic.three_gas_lines(30000, 1480.0, 1540.0, seed=9), 1480.0, 1540.0)
    lv = synthetic.perturbed_levels(synthetic.logp_levels(9), 2, seed=6)
    vmr = {g: lv[g] for g in ("H2O", "CO2", "O3")}
    nu, tb = lbl.transmittance_batch(sd, lv["p"], lv["t"], vmr, 1500.0, 1505.0, mu_view=0.8)
    centres, ch = lbl.transmittance_batch(sd, lv["p"], lv["t"], vmr, 1500.0, 1505.0, mu_view=0.8,
                                          channel_width_cm1=0.25)
    assert ch.shape == (2, 20) and centres.size == 20
    ref = tb[:, :20 * 250].reshape(2, 20, 250).mean(axis=2)
    np.testing.assert_allclose(ch, ref, rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(centres, nu[:5000].reshape(20, 250).mean(axis=1), rtol=0, atol=1e-9)


def test_channel_means_against_oracle(cuda):
    """Device channel means (box averages of T over 200 grid points) against the oracle's
    float64 transmittance averaged on the host, per profile and view cosine."""
    lo, hi, cutoff, step = 1500.0, 1503.0, 3.0, 0.001
    sd = synthetic.restrict(synthetic.three_gas_lines(4000, lo - cutoff - 1, hi + cutoff + 1, seed=21),
                            lo - cutoff - 1, hi + cutoff + 1)
    lv = synthetic.perturbed_levels(synthetic.logp_levels(7), 2, seed=8)
    for g in ("H2O", "CO2", "O3"):                         # thin the column to optical depths of order 1
        lv[g] = lv[g] * 2e-5
    mu = np.array([0.9, 0.6])
    nu = restate.grid(lo, hi, step)
    width = 200
    n_ch = nu.size // width
    ref = np.empty((2, n_ch))
    for i in range(2):
        inp = oracle_inputs(sd, synthetic.profile_from_levels(lv, i))
        od = restate.optical_depth(nu, inp["lines"], inp["tips"], inp["masses"], inp["p_atm"], inp["t_layer"],
                                   inp["vmr_layer"], inp["col"], cutoff, 2.0)
        ref[i] = restate.transmittance(nu, od, mu[i])[: n_ch * width].reshape(n_ch, width).mean(axis=1)
    assert 0.01 < ref.min() and ref.max() < 0.95             # neither saturated nor transparent
    for precision in ("fp64", "fp32"):
        centres, ch = lbl.transmittance_batch(sd, lv["p"], lv["t"], {g: lv[g] for g in ("H2O", "CO2", "O3")},
                                              lo, hi, step_cm1=step, line_cutoff_cm1=cutoff, mu_view=mu,
                                              precision=precision, channel_width_cm1=width * step)
        assert ch.shape == (2, n_ch)
        assert np.max(np.abs(ch - ref)) <= TOL[precision]["dT"], precision
        np.testing.assert_allclose(centres, nu[: n_ch * width].reshape(n_ch, width).mean(axis=1), rtol=0, atol=1e-9)


def test_fp32_bitwise_reproducible_with_overlapping_near_zones(cuda):
    """300 lines per cm^-1 (near zones overlap): repeated launches and a batch of
    profiles give the same float32 optical depth bit for bit, for both precisions."""
    sd = synthetic.restrict(synthetic.three_gas_lines(6000, 1492, 1512, seed=3), 1492, 1512)
    lv = synthetic.perturbed_levels(synthetic.logp_levels(6), 3, seed=77)
    gases = ["H2O", "CO2", "O3"]
    grid = engine.make_grid(1500.0, 1503.0, 0.001, 2.0)

    def job(sl):
        li = engine.LayerInput(gases=gases, levels_p=lv["p"][sl], levels_t=lv["t"][sl],
                               levels_vmr=np.stack([lv[g][sl] for g in gases], axis=1))
        return engine.Job(sd, li, grid, 25.0)

    single, both = job(slice(0, 1)), job(slice(0, 3))
    for precision in ("fp32", "fp64"):
        a = single.run(precision, deterministic=True).od[0]
        b = single.run(precision, deterministic=True).od[0]
        c = both.run(precision, deterministic=True).od[0]
        assert torch.equal(a, b) and torch.equal(a, c), precision
    # the default float32 sums (atomic near-zone corrections) agree to rounding
    d = both.run("fp32").od[0]
    assert torch.max(torch.abs(d - a)).item() <= 1e-6 * torch.max(torch.abs(a)).item()
    with pytest.raises(ValueError, match="deterministic"):
        single.run("fp32-direct", deterministic=True)


def test_wavenumber_shards_equal_the_full_spectrum(cuda):
    """Reference tiles computed in three ranges (shards) give the full spectrum bit for bit."""
    from pylblrtm_b200 import shard
    sd = synthetic.restrict(synthetic.three_gas_lines(30000, 1480.0, 1540.0, seed=9), 1480.0, 1540.0)
    prof = synthetic.profile_from_levels(synthetic.logp_levels(9))
    sd = synthetic.scale_strengths(sd, 1e-4)
    grid = engine.make_grid(1500.0, 1507.3, 0.001, 2.0)          # 4 tiles, the last one partial
    job = engine.Job(sd, engine.layer_input_from_profile(prof), grid, 25.0)
    full = job.run("fp32", mu=[0.8], want_od=True, want_trans=True, deterministic=True)
    pieces = [job.run("fp32", mu=[0.8], want_od=True, want_trans=True, deterministic=True, tiles=t)
              for t in ((0, 1), (1, 2), (3, 1))]
    assert torch.equal(torch.cat([p.trans for p in pieces], dim=1), full.trans)
    assert torch.equal(torch.cat([p.od for p in pieces], dim=2), full.od)
    nu, t = shard.compute_transmittance_sharded(sd, prof, 1500.0, 1507.3, mu_view=0.8)
    _, t_ref = lbl.compute_transmittance(sd, prof, 1500.0, 1507.3, mu_view=0.8, deterministic=True)
    assert np.array_equal(t, t_ref) and t.min() < 0.99
    # shard jobs: each range from only the lines of its window, bit for bit the full job's
    for first, count in ((0, 1), (1, 2), (3, 1)):
        sj = shard.shard_job(sd, prof, grid, 25.0, first, count)
        assert sj.n_bound < job.n_bound
        piece = sj.run("fp32", mu=[0.8], want_od=True, want_trans=True, deterministic=True, tiles=(first, count))
        ref = job.run("fp32", mu=[0.8], want_od=True, want_trans=True, deterministic=True, tiles=(first, count))
        assert torch.equal(piece.od, ref.od) and torch.equal(piece.trans, ref.trans)
    with pytest.raises(ValueError, match="outside the grid"):
        job.run("fp32", tiles=(3, 2))
    with pytest.raises(ValueError, match="tiles needs"):
        job.run("fp64", tiles=(0, 1))


@pytest.mark.parametrize("tile,step", [(2.0, 0.001), (5.0, 0.001), (0.05, 0.001), (0.3, 0.0025)])
def test_inner_ranges_select_every_inner_line(cuda, tile, step, monkeypatch):
    """The multi-level sum with the per-tile inner-line ranges does exactly the work of
    the same sum scanning every candidate line of the tile (inner = NULL): equal
    reference-rule evaluation counts and equal level-2 / level-3 / near-zone counts, so
    no inner line is lost, and optical depths equal to float rounding (the scans group
    lines into different 256-line rounds). Pressure shifts are 40x the synthetic ones;
    tiles of one chunk, three chunks, and tiles too small for level 1."""
    sd = synthetic.restrict(synthetic.three_gas_lines(20000, 1490.0, 1520.0, seed=4), 1490.0, 1520.0)
    lines = {k: v.copy() for k, v in sd.lines.items()}
    lines["shift"] = lines["shift"] * 40.0
    sd = SpectralData(lines, dict(sd.tips), dict(sd.molar_masses), sd.molecule)
    lv = synthetic.perturbed_levels(synthetic.logp_levels(7), 2, seed=8)
    gases = ["H2O", "CO2", "O3"]
    li = engine.LayerInput(gases=gases, levels_p=lv["p"], levels_t=lv["t"],
                           levels_vmr=np.stack([lv[g] for g in gases], axis=1))
    job = engine.Job(sd, li, engine.make_grid(1500.0, 1510.3, step, tile), 5.0)
    with_inner = job.run("fp32", deterministic=True, count_evals=True)
    real_call = _lib.call

    def no_inner(name, *args):
        if name == "lbl_tau_tiles_ml_f32":
            args = args[:3] + (0,) + args[4:]
        return real_call(name, *args)

    monkeypatch.setattr(_lib, "call", no_inner)
    scan_all = job.run("fp32", deterministic=True, count_evals=True)
    assert with_inner.evals == scan_all.evals and with_inner.work_split == scan_all.work_split
    rel = ((with_inner.od - scan_all.od).abs() / scan_all.od.abs().clamp_min(1e-30)).max().item()
    assert rel <= 2e-6, rel


def test_batch_of_zero_profiles(cuda):
    """A rank whose share of a sharded batch is empty gets an empty [0, n] result."""
    from pylblrtm_b200 import batch
    sd = synthetic.restrict(synthetic.three_gas_lines(3000, 990.0, 1030.0, seed=3), 990.0, 1030.0)
    lv = synthetic.perturbed_levels(synthetic.logp_levels(9), 2, seed=5)
    vmr = {g: lv[g][:0] for g in ("H2O", "CO2", "O3")}
    nu, t = batch.transmittance_batch(sd, lv["p"][:0], lv["t"][:0], vmr, 1000.0, 1003.0)
    assert t.shape == (0, nu.size) and nu.size == 3001
    ax, ch = batch.transmittance_batch(sd, lv["p"][:0], lv["t"][:0], vmr, 1000.0, 1003.0, channel_width_cm1=0.25,
                                       as_numpy=False)
    assert tuple(ch.shape) == (0, ax.size) and ch.is_cuda


@pytest.mark.parametrize("tile", [2.06, 1.05])
def test_tiles_just_over_a_chunk_keep_float32_accuracy(cuda, tile):
    """Tiles a few points longer than the longest chunk (2,048 points for the forward, 1,024
    for the Jacobian) are cut into near-equal chunks, not into a full chunk plus a sliver: a
    sliver of a dozen points has no far-field level, so all of the ~5,000 lines of its window
    were summed directly in float32 there (relative od error 1e-5 against float64). The
    forward and the Jacobian's od stay within 3e-6 of the float64 engine."""
    sd = synthetic.restrict(synthetic.three_gas_lines(), 975.0, 1075.0)
    job = engine.Job(sd, engine.layer_input_from_profile(synthetic.logp_profile()),
                     engine.make_grid(1000.0, 1050.0, 0.001, tile), 25.0)
    od64 = job.run("fp64", want_od=True).od[0].double()
    rel = lambda a: ((a.double() - od64).abs() / od64.abs().clamp_min(1e-300)).max().item()
    assert rel(job.run("fp32", want_od=True).od[0]) <= 3e-6
    assert rel(job.jacobian("H2O", deterministic=True)[0][0]) <= 3e-6
