"""YAML-driven runner (drop-in for ``pylblrtm/config.py``).

Same defaults, merge, validation, result container and writers as the
reference (``config.py:23-319``); the optical depth comes from the GPU engine.
An optional ``engine`` section (ignored by the reference) selects the
precision: ``engine: {precision: fp32|fp32-direct|fp64, deterministic: false|true}``.
"""

from __future__ import annotations

import copy
from dataclasses import dataclass, field
from pathlib import Path
from typing import Optional, Union

import numpy as np

from . import engine
from .atmosphere import AtmosphericProfile
from .forward import DEFAULT_PRECISION
from .spectral_data import SpectralData

_DEFAULTS: dict = {
    "spectral": {"nu_min_cm1": 700.0, "nu_max_cm1": 750.0, "step_cm1": 0.001},
    "calculation": {"mu_view": 1.0, "line_cutoff_cm1": 25.0, "tile_width_cm1": 2.0},
    "output": {
        "transmittance": True,
        "optical_depth": False,
        "optical_depth_layers": False,
        "save": {"enabled": False, "path": "results/", "format": "npz", "prefix": "forward"},
    },
}


def _deep_merge(base: dict, override: dict) -> dict:
    """Recursively merge ``override`` into a copy of ``base``."""
    result = dict(base)
    for key, value in override.items():
        if key in result and isinstance(result[key], dict) and isinstance(value, dict):
            result[key] = _deep_merge(result[key], value)
        else:
            result[key] = value
    return result


def load_config(source: Union[str, Path, dict]) -> dict:
    """Config from a YAML file or dict, merged over the defaults and validated."""
    if isinstance(source, dict):
        raw = source
    else:
        try:
            import yaml
        except ImportError:
            raise ImportError("PyYAML is required to load YAML config files. "
                              "Install it with:  pip install pyyaml") from None
        path = Path(source)
        if not path.exists():
            raise FileNotFoundError(f"Config file not found: {path}")
        with open(path, "r", encoding="utf-8") as fh:
            raw = yaml.safe_load(fh) or {}
    cfg = _deep_merge(_DEFAULTS, raw)
    _validate(cfg)
    return cfg


def _validate(cfg: dict) -> None:
    sp, ca, out = cfg["spectral"], cfg["calculation"], cfg["output"]
    if sp["nu_min_cm1"] >= sp["nu_max_cm1"]:
        raise ValueError("spectral.nu_min_cm1 must be strictly less than nu_max_cm1")
    if sp["step_cm1"] <= 0:
        raise ValueError("spectral.step_cm1 must be positive")
    if ca["line_cutoff_cm1"] <= 0:
        raise ValueError("calculation.line_cutoff_cm1 must be positive")
    if not (0.0 < ca["mu_view"] <= 1.0):
        raise ValueError("calculation.mu_view must be in (0, 1]")
    if not any([out["transmittance"], out["optical_depth"], out["optical_depth_layers"]]):
        raise ValueError("At least one output must be enabled: "
                         "transmittance, optical_depth, or optical_depth_layers")
    fmt = out["save"]["format"]
    if fmt not in {"npz", "csv", "txt"}:
        raise ValueError(f"output.save.format must be 'npz', 'csv', or 'txt'; got '{fmt}'")
    det = cfg.get("engine", {}).get("deterministic", False)
    if not isinstance(det, bool):
        raise ValueError(f"engine.deterministic must be true or false; got '{det}'")
    prec = cfg.get("engine", {}).get("precision", DEFAULT_PRECISION)
    if prec not in engine.PRECISIONS:
        raise ValueError(f"engine.precision must be one of {engine.PRECISIONS}; got '{prec}'")


@dataclass
class ForwardResult:
    """Output of :func:`run_forward`; unrequested fields stay ``None``."""

    wavenumber_cm1: np.ndarray
    config: dict
    transmittance: Optional[np.ndarray] = field(default=None)
    optical_depth: Optional[np.ndarray] = field(default=None)
    optical_depth_layers: Optional[np.ndarray] = field(default=None)

    def save(self, path: Optional[str] = None, fmt: Optional[str] = None,
             prefix: Optional[str] = None) -> Path:
        """Write the outputs; arguments default to ``output.save.*`` of the config."""
        sv = self.config["output"]["save"]
        return _write(self, path=path or sv["path"], fmt=fmt or sv["format"], prefix=prefix or sv["prefix"])

    def __repr__(self) -> str:
        nu = self.wavenumber_cm1
        parts = []
        if self.transmittance is not None:
            parts.append("transmittance")
        if self.optical_depth is not None:
            parts.append("optical_depth")
        if self.optical_depth_layers is not None:
            parts.append(f"optical_depth_layers{list(self.optical_depth_layers.shape)}")
        return (f"ForwardResult(nu=[{nu[0]:.2f}, {nu[-1]:.2f}] cm-1 | step={nu[1]-nu[0]:.4g} cm-1 | "
                f"outputs=[{', '.join(parts)}])")


def run_forward(spectral_data: SpectralData, profile: AtmosphericProfile,
                config: Union[str, Path, dict]) -> ForwardResult:
    """Forward model driven by a YAML file or dict (``pylblrtm/config.py:196-279``)."""
    if not isinstance(spectral_data, SpectralData):
        raise TypeError("spectral_data must be a SpectralData instance")
    if not isinstance(profile, AtmosphericProfile):
        raise TypeError("profile must be an AtmosphericProfile instance")
    cfg = load_config(config)
    sp, ca, out = cfg["spectral"], cfg["calculation"], cfg["output"]
    grid = engine.make_grid(float(sp["nu_min_cm1"]), float(sp["nu_max_cm1"]), float(sp["step_cm1"]),
                            float(ca["tile_width_cm1"]))
    mu = float(ca["mu_view"])
    nu = engine.grid_async(grid)
    res = engine.optical_depth(
        spectral_data, engine.layer_input_from_profile(profile), grid, float(ca["line_cutoff_cm1"]),
        precision=cfg.get("engine", {}).get("precision", DEFAULT_PRECISION), mu=[mu],
        deterministic=cfg.get("engine", {}).get("deterministic", False),
        want_od=bool(out["optical_depth_layers"]), want_tau=bool(out["optical_depth"]),
        want_trans=bool(out["transmittance"]), warn_level=3)
    result = ForwardResult(wavenumber_cm1=nu.result(), config=cfg)
    if out["transmittance"]:
        result.transmittance = engine.to_host(res.trans[0])
    if out["optical_depth"]:
        result.optical_depth = engine.to_host(res.tau[0])        # vertical, not divided by mu
    if out["optical_depth_layers"]:
        result.optical_depth_layers = engine.to_host(res.od[0].double())
    if out["save"]["enabled"]:
        result.save()
    return result


def _write(result: ForwardResult, path: str, fmt: str, prefix: str) -> Path:
    out_dir = Path(path)
    out_dir.mkdir(parents=True, exist_ok=True)
    if fmt == "npz":
        arrays: dict = {"wavenumber_cm1": result.wavenumber_cm1}
        for name in ("transmittance", "optical_depth", "optical_depth_layers"):
            v = getattr(result, name)
            if v is not None:
                arrays[name] = v
        out_path = out_dir / f"{prefix}.npz"
        np.savez(out_path, **arrays)
    else:
        sep = "," if fmt == "csv" else "\t"
        cols, headers = [result.wavenumber_cm1], ["wavenumber_cm1"]
        for name in ("transmittance", "optical_depth"):
            v = getattr(result, name)
            if v is not None:
                cols.append(v)
                headers.append(name)
        out_path = out_dir / f"{prefix}.{fmt}"
        np.savetxt(out_path, np.column_stack(cols), delimiter=sep, header=sep.join(headers), comments="")
    print(f"Saved: {out_path}")
    return out_path
