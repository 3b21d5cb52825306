"""The reference-side binding: the GPU ``_build_optical_depth`` patched into a module
shaped like ``pylblrtm.forward`` and driven with objects shaped like the reference's own.

A maintainer who keeps the reference package and routes only its hot loop to the GPU
replaces ``pylblrtm.forward._build_optical_depth`` (``pylblrtm/forward.py:157``, also
imported by ``pylblrtm/config.py:19`` and called at ``config.py:253``) with
``pylblrtm_b200.forward._build_optical_depth``. The reference calls it with its own
``_Layers`` dataclass (``pylblrtm/atmosphere.py:22-35``) and its own ``SpectralData``
(``pylblrtm/spectral_data.py:14-78``). Neither type is importable where the GPU tests
run, so these tests use stand-ins with the reference's field names and no others, and
a module whose ``compute_transmittance`` body does what ``forward.py:141-151`` does
around the call (grid, layers, optical depth, ``exp(-sum od / mu)``). Results are
checked against the golden vectors made by running the reference itself.
"""

import dataclasses
import types
import warnings
from typing import Dict, Optional, Tuple

import numpy as np
import pytest

from conftest import golden_case
from oracle import restate

pytestmark = pytest.mark.gpu


@dataclasses.dataclass
class RefLayers:
    """Fields of the reference's ``_Layers`` (atmosphere.py:22-35), nothing else."""
    pressure_atm: np.ndarray
    temperature_k: np.ndarray
    vmr: Dict[str, np.ndarray]
    column_cm2: Dict[str, np.ndarray]

    @property
    def n_layers(self) -> int:
        return len(self.pressure_atm)


@dataclasses.dataclass
class RefSpectralData:
    """Fields of the reference's ``SpectralData`` (spectral_data.py:36-39) and its Q()."""
    lines: Dict[str, np.ndarray]
    tips: Dict[tuple, Tuple[np.ndarray, np.ndarray]]
    molar_masses: Dict[tuple, float]
    molecule: Optional[str] = None

    def Q(self, T, mol_id, iso_id):
        t, q = self.tips[(int(mol_id), int(iso_id))]
        return np.interp(T, t, q)


def _reference_shaped_module():
    """A stand-in for ``pylblrtm.forward`` whose compute path calls the module-level
    ``_build_optical_depth`` the way ``forward.py:141-151`` does."""
    mod = types.ModuleType("pylblrtm_forward_standin")

    def _build_optical_depth(nu, sd, layers, cutoff, tile):   # replaced by the patch below
        raise AssertionError("the unpatched stand-in must not run")

    def compute_transmittance(sd, levels, nu_min, nu_max, step, cutoff, tile, mu):
        n = int(np.ceil((nu_max - nu_min) / step)) + 1
        nu = nu_min + np.arange(n) * step
        p, t, v, c = restate.build_layers(*levels)
        layers = RefLayers(pressure_atm=p, temperature_k=t, vmr=v, column_cm2=c)
        od = mod._build_optical_depth(nu, sd, layers, cutoff, tile)
        return nu, np.exp(-od.sum(axis=0) / mu), od

    mod._build_optical_depth = _build_optical_depth
    mod.compute_transmittance = compute_transmittance
    return mod


@pytest.mark.parametrize("name", ["edge_mix", "tile0.5", "three_gas_win1500_thin", "co2_band_mid"])
def test_patched_reference_module_matches_golden(cuda, name):
    from pylblrtm_b200.forward import _build_optical_depth as gpu_od
    sd, prof, prm, data = golden_case(name)
    ref_sd = RefSpectralData(dict(sd.lines), dict(sd.tips), dict(sd.molar_masses), sd.molecule)
    fwd = _reference_shaped_module()
    fwd._build_optical_depth = gpu_od                      # the maintainer's patch (float32 engine)
    with warnings.catch_warnings(record=True) as wl:
        warnings.simplefilter("always")
        nu, T, od = fwd.compute_transmittance(ref_sd, (prof.pressure_hpa, prof.temperature_k, prof.vmr),
                                              prm["nu_min"], prm["nu_max"], prm["step"], prm["cutoff"],
                                              prm["tile"], prm["mu"])
    assert od.dtype == np.float64 and od.shape == (prof.n_levels - 1, int(data["n_nu"]))
    assert np.max(np.abs(T - data["T"])) <= 1e-5
    tau = od.sum(axis=0)
    m = data["tau"] > 1e-300
    assert np.max(np.abs(tau - data["tau"])[m] / data["tau"][m]) <= 2e-5
    if "od_layers" in data:
        ref = data["od_layers"]
        mm = np.abs(ref) > 1e-300
        assert np.max(np.abs(od - ref)[mm] / np.abs(ref)[mm]) <= 3e-5
    assert sorted(str(w.message) for w in wl) == sorted(m_ for m_ in data["warnings"].tolist() if m_)


def test_patched_module_float64_engine(cuda):
    """The same patch with the float64 engine selected (the keyword the GPU version adds)."""
    import functools
    from pylblrtm_b200.forward import _build_optical_depth as gpu_od
    sd, prof, prm, data = golden_case("tile2.0")
    ref_sd = RefSpectralData(dict(sd.lines), dict(sd.tips), dict(sd.molar_masses), sd.molecule)
    fwd = _reference_shaped_module()
    fwd._build_optical_depth = functools.partial(gpu_od, precision="fp64")
    _, T, od = fwd.compute_transmittance(ref_sd, (prof.pressure_hpa, prof.temperature_k, prof.vmr),
                                         prm["nu_min"], prm["nu_max"], prm["step"], prm["cutoff"], prm["tile"],
                                         prm["mu"])
    assert np.max(np.abs(T - data["T"])) <= 1e-6
    ref = data["od_layers"]
    mm = np.abs(ref) > 1e-300
    assert np.max(np.abs(od - ref)[mm] / np.abs(ref)[mm]) <= 1e-9
