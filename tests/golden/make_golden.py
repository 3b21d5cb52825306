"""Generate golden vectors by running the REFERENCE forward model (PyLBLRTM).

Run in a container where the reference source is present:

    python tests/golden/make_golden.py --reference <source tree of the reference package>

Each case builds seeded synthetic inputs with ``pylblrtm_b200.synthetic``,
converts them to the reference's own SpectralData / AtmosphericProfile objects
and calls the reference's public functions (``compute_transmittance``,
``run_forward``) or its internal ``_build_optical_depth``. Outputs are written as
compressed ``.npz`` files next to this script, with a SHA-256 of the inputs so
the tests can detect a change in the generators.
"""

from __future__ import annotations

import argparse
import hashlib
import multiprocessing as mp
import os
import sys
import time
import warnings

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.abspath(os.path.join(HERE, "..", "..")))

from pylblrtm_b200 import synthetic as syn  # noqa: E402
from pylblrtm_b200.spectral_data import LINE_KEYS  # noqa: E402


def input_digest(sd, prof) -> str:
    h = hashlib.sha256()
    for k in LINE_KEYS:
        h.update(np.ascontiguousarray(sd.lines[k]).tobytes())
    for key in sorted(sd.tips):
        h.update(repr(key).encode())
        for a in sd.tips[key]:
            h.update(np.ascontiguousarray(a).tobytes())
    h.update(repr(sorted(sd.molar_masses.items())).encode())
    h.update(prof.pressure_hpa.tobytes())
    h.update(prof.temperature_k.tobytes())
    for g in sorted(prof.vmr):
        h.update(g.encode())
        h.update(prof.vmr[g].tobytes())
    return h.hexdigest()


def cases():
    """name -> (builder of (sd, profile), nu_min, nu_max, step, cutoff, tile, mu, keep_layers)."""
    c = {}
    c["co2_band_full"] = (lambda: (syn.co2_band(), syn.us_standard_atmosphere(["CO2"])),
                          700.0, 750.0, 0.001, 25.0, 2.0, 1.0, False)
    c["co2_band_mid"] = (lambda: (syn.scale_strengths(syn.co2_band(), 1e-3),
                                  syn.us_standard_atmosphere(["CO2"])),
                         700.0, 750.0, 0.001, 25.0, 2.0, 1.0, False)
    c["co2_band_top3"] = (lambda: (syn.co2_band(), _top_levels(syn.us_standard_atmosphere(["CO2"]), 4)),
                          700.0, 750.0, 0.001, 25.0, 2.0, 1.0, False)
    for lo in (600.0, 1500.0, 2495.0):
        c[f"three_gas_win{int(lo)}"] = (lambda: (syn.three_gas_lines(), syn.logp_profile()),
                                        lo, lo + 5.0, 0.001, 25.0, 2.0, 0.8, False)
    c["three_gas_win1500_thin"] = (lambda: (syn.scale_strengths(syn.three_gas_lines(), 1e-5),
                                            syn.logp_profile()),
                                   1500.0, 1505.0, 0.001, 25.0, 2.0, 0.8, False)
    for tile in (2.0, 0.5):
        c[f"tile{tile}"] = (lambda: (syn.co2_band(300, 700.0, 720.0, seed=11),
                                     _top_levels(syn.us_standard_atmosphere(["CO2"]), 6)),
                            705.0, 712.0, 0.001, 1.0, tile, 1.0, True)
    c["edge_mix"] = (_edge_case, 700.0, 703.0, 0.002, 5.0, 0.7, 0.6, True)
    c["coarse_step"] = (lambda: (syn.co2_band(400, 700.0, 760.0, seed=5),
                                 syn.us_standard_atmosphere(["CO2", "H2O"])),
                        701.3, 758.9, 0.01, 25.0, 2.0, 0.9, False)
    return c


def _top_levels(prof, n):
    from pylblrtm_b200.atmosphere import AtmosphericProfile
    return AtmosphericProfile(prof.pressure_hpa[:n], prof.temperature_k[:n],
                              {g: v[:n] for g, v in prof.vmr.items()})


def _edge_case():
    """Lines and tables that exercise every skip / fallback branch of the reference."""
    from pylblrtm_b200.atmosphere import AtmosphericProfile
    from pylblrtm_b200.spectral_data import SpectralData
    rng = np.random.default_rng(99)
    n = 240
    lines = {
        "nu0": np.concatenate([rng.uniform(697.0, 706.0, n - 40), [693.0, 699.9, 703.05, 708.1],
                               rng.uniform(699.0, 704.0, 36)]),
        "Sref": 10.0 ** rng.uniform(-29, -23, n),
        "g_air": rng.uniform(0.01, 0.09, n),
        "g_self": rng.uniform(0.05, 0.12, n),
        "Elow": rng.uniform(0.0, 4000.0, n),
        "n_air": rng.uniform(-0.3, 0.9, n),          # negative exponents included
        "shift": rng.uniform(-0.01, 0.006, n),       # both signs
        "mol_id": np.empty(n, np.int32),
        "iso_id": np.ones(n, np.int32),
    }
    groups = np.array([2, 2, 1, 3, 6, 99, 7])        # 6=CH4 absent from profile, 99 unknown, 7 no mass
    lines["mol_id"][:] = groups[rng.integers(0, groups.size, n)]
    lines["iso_id"][(lines["mol_id"] == 2) & (rng.uniform(size=n) < 0.5)] = 2
    tips = {
        (2, 1): syn.tips_power_law(286.0),
        (2, 2): (np.arange(200.0, 251.0), 570.0 * (np.arange(200.0, 251.0) / 296.0) ** 1.5),  # clamps
        (1, 1): syn.tips_power_law(174.0),
        (3, 1): syn.tips_power_law(3483.0, 150.0, 400.0, 2.5),
        (6, 1): syn.tips_power_law(590.0),
        (7, 1): syn.tips_power_law(215.0),
    }
    masses = {(2, 1): 43.99, (2, 2): 44.99, (1, 1): 18.01, (3, 1): 47.98, (6, 1): 16.03}
    sd = SpectralData(lines, tips, masses, None)
    p = np.array([0.5, 3.0, 20.0, 150.0, 500.0, 1013.25])
    t = np.array([265.0, 240.0, 215.0, 230.0, 270.0, 295.0])
    vmr = {
        "CO2": np.full(6, 415e-6),
        "H2O": np.array([0.0, 0.0, 3e-6, 1e-4, 4e-3, 1.5e-2]),    # col == 0 in top layer
        "O3": np.array([3e-6, 6e-6, 5e-6, 3e-7, 5e-8, 3e-8]),
        "O2": np.full(6, 0.2095),
    }
    return sd, AtmosphericProfile(p, t, vmr)


def to_reference(sd, prof):
    from pylblrtm.atmosphere import AtmosphericProfile as RP
    from pylblrtm.spectral_data import SpectralData as RSD
    rsd = RSD({k: np.asarray(v).copy() for k, v in sd.lines.items()},
              {k: (a.copy(), b.copy()) for k, (a, b) in sd.tips.items()},
              dict(sd.molar_masses), sd.molecule)
    return rsd, RP(prof.pressure_hpa.copy(), prof.temperature_k.copy(),
                   {g: v.copy() for g, v in prof.vmr.items()})


def run_case(args):
    name, ref_root = args
    sys.path.insert(0, ref_root)
    from pylblrtm.config import run_forward
    builder, lo, hi, step, cutoff, tile, mu, keep_layers = cases()[name]
    sd, prof = builder()
    rsd, rprof = to_reference(sd, prof)
    cfg = {"spectral": {"nu_min_cm1": lo, "nu_max_cm1": hi, "step_cm1": step},
           "calculation": {"mu_view": mu, "line_cutoff_cm1": cutoff, "tile_width_cm1": tile},
           "output": {"transmittance": True, "optical_depth": True,
                      "optical_depth_layers": keep_layers}}
    t0 = time.time()
    with warnings.catch_warnings(record=True) as wlist:
        warnings.simplefilter("always")
        res = run_forward(rsd, rprof, cfg)
    dt = time.time() - t0
    out = {
        "nu_min": lo, "nu_max": hi, "step": step, "cutoff": cutoff, "tile": tile, "mu": mu,
        "n_nu": res.wavenumber_cm1.size,
        "tau": res.optical_depth, "T": res.transmittance,
        "warnings": np.array([str(w.message) for w in wlist] or [""]),
        "input_sha256": input_digest(sd, prof),
        "seconds": dt,
    }
    if keep_layers:
        out["od_layers"] = res.optical_depth_layers
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    return name, dt


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="source tree that holds the pylblrtm package")
    ap.add_argument("--only", nargs="*")
    ap.add_argument("--jobs", type=int, default=os.cpu_count())
    a = ap.parse_args()
    names = a.only or list(cases())
    ctx = mp.get_context("spawn")
    with ctx.Pool(min(a.jobs, len(names))) as pool:
        for name, dt in pool.imap_unordered(run_case, [(n, a.reference) for n in names]):
            print(f"{name}: {dt:.1f} s", flush=True)


if __name__ == "__main__":
    main()
