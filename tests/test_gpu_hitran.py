"""A line list read from a HITRAN .par file (tests/golden/hitran/clean.par) through from_files,
run by the GPU engines and compared with the float64 oracle on the same parsed data."""

import os

import numpy as np
import pytest

from conftest import GOLDEN_DIR, oracle_inputs
from oracle import restate
import pylblrtm_b200 as lbl
from pylblrtm_b200 import hitran_io

pytestmark = pytest.mark.gpu

HIT = os.path.join(GOLDEN_DIR, "hitran")


@pytest.mark.parametrize("precision,dT,rtau", [("fp32", 1e-5, 2e-5), ("fp64", 1e-6, 1e-9)])
def test_par_file_through_the_engine(cuda, precision, dT, rtau):
    par = os.path.join(HIT, "clean.par")
    d = hitran_io.par_to_dict(par)
    present = sorted(set(zip(d["mol_id"].tolist(), d["iso_id"].tolist())))
    masses = {k: {1: 18.01, 2: 43.99, 3: 47.98}[k[0]] + 1.0 * (k[1] - 1) for k in present}
    sd = lbl.from_files(par, {k: os.path.join(HIT, "tips_a.txt") for k in present}, molar_masses=masses)
    # the file's strengths reach 1e-18; scale them so the window is not saturated
    sd = lbl.SpectralData({**sd.lines, "Sref": sd.lines["Sref"] * 1e-3}, sd.tips, sd.molar_masses, sd.molecule)
    prof = lbl.us_standard_atmosphere(["H2O", "CO2", "O3"])
    lo, hi, step = 1000.0, 1010.0, 0.002
    nu, T = lbl.compute_transmittance(sd, prof, lo, hi, step_cm1=step, precision=precision)
    inp = oracle_inputs(sd, prof)
    nu_ref = restate.grid(lo, hi, step)
    od = restate.optical_depth(nu_ref, inp["lines"], inp["tips"], inp["masses"], inp["p_atm"], inp["t_layer"],
                               inp["vmr_layer"], inp["col"])
    T_ref = restate.transmittance(nu_ref, od)
    tau_ref = od.sum(0)
    assert np.array_equal(nu, nu_ref)
    assert np.max(np.abs(T - T_ref)) <= dT
    m = tau_ref > 1e-12
    assert np.max(np.abs(-np.log(T[m]) - tau_ref[m]) / tau_ref[m]) <= rtau
    assert T.min() < 0.99 and T.max() > 0.01          # the window is neither empty nor saturated
