"""Shared test helpers: the `gpu` marker, golden-vector loading and case builders."""

import importlib.util
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN_DIR = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


def golden_module():
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN_DIR, "make_golden.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def golden_case(name):
    """(inputs, case parameters, stored reference outputs) of one golden vector."""
    mg = golden_module()
    builder, lo, hi, step, cutoff, tile, mu, keep = mg.cases()[name]
    sd, prof = builder()
    data = dict(np.load(os.path.join(GOLDEN_DIR, f"{name}.npz")))
    assert str(data["input_sha256"]) == mg.input_digest(sd, prof), \
        f"synthetic inputs of {name} changed; regenerate tests/golden"
    params = dict(nu_min=lo, nu_max=hi, step=step, cutoff=cutoff, tile=tile, mu=mu)
    return sd, prof, params, data


def oracle_inputs(sd, prof):
    """Plain arrays for oracle.restate from package objects."""
    from oracle import restate
    p, t, v, c = restate.build_layers(prof.pressure_hpa, prof.temperature_k, prof.vmr)
    return dict(lines={k: np.asarray(a) for k, a in sd.lines.items()}, tips=sd.tips,
                masses=sd.molar_masses, p_atm=p, t_layer=t, vmr_layer=v, col=c)


SMALL_GOLDEN = ["edge_mix", "tile2.0", "tile0.5", "coarse_step"]
ALL_GOLDEN = SMALL_GOLDEN + ["co2_band_top3", "co2_band_mid", "co2_band_full", "three_gas_win600",
                             "three_gas_win1500", "three_gas_win2495", "three_gas_win1500_thin"]


@pytest.fixture(scope="session")
def cuda():
    """The CUDA device; GPU tests fail (not skip) when it is missing."""
    import torch
    assert torch.cuda.is_available(), "GPU test run without a CUDA device"
    from pylblrtm_b200 import _lib
    _lib.load()
    return torch.device("cuda", 0)
