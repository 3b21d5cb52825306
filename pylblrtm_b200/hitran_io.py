"""HITRAN text inputs: ``.par`` line lists and TIPS tables (drop-in for the readers of
``pylblrtm/hitran_manager.py`` and ``pylblrtm/data_loader.py:92-175``).

``par_to_dict`` parses with the native reader ``liblblio.so`` (``include/lblio.h``,
``csrc/hitran_par.cpp``), which follows ``hitran_manager.py:816-872`` character for
character; this module assembles the reference's columns (which can differ in length
after a malformed line, as the reference appends field by field), its warnings and its
errors. Lines containing non-ASCII bytes (rare) and malformed lines are re-read here
with Python's own ``int``/``float``, so values and warning texts are the reference's.
``txt_to_tips`` (``hitran_manager.py:917-963``) and ``from_files`` are host Python, as
in the reference. Nothing here touches the GPU.
"""

from __future__ import annotations

import ctypes
import logging
import os
import re
from pathlib import Path
from typing import Dict, Optional, Tuple, Union

import numpy as np

from .hitran_ids import MOLECULE_IDS
from .spectral_data import SpectralData

logger = logging.getLogger(__name__)

PAR_SHORT, PAR_NONASCII = -1, -2
COLUMNS = ("mol_id", "iso_id", "nu0", "Sref", "g_air", "g_self", "Elow", "n_air", "shift")
_SLICES = ((0, 2), (2, 3), (3, 15), (15, 25), (35, 40), (40, 45), (45, 55), (55, 59), (59, 67))
_ID_TO_MOL = {v: k for k, v in MOLECULE_IDS.items()}



class HITRANDataError(ValueError):
    """Malformed or empty HITRAN data (hitran_manager.py:134)."""


def _lib() -> ctypes.CDLL:
    from . import _lib as lib_mod
    return lib_mod.load_host()


def _python_fields(raw: str):
    """The reference's per-line conversion (hitran_manager.py:847-857): values converted
    before the first failure, and the failure."""
    out = []
    for k, (a, b) in enumerate(_SLICES):
        try:
            out.append(int(raw[a:b]) if k < 2 else float(raw[a:b]))
        except ValueError as exc:
            return out, exc
    return out, None


def _split_lines(data: bytes):
    """Lines of the file under universal newlines (\\r and \\n are single bytes in UTF-8)."""
    parts = re.split(rb"\r\n|\r|\n", data)
    if parts and parts[-1] == b"":
        parts.pop()
    return parts


def par_to_dict(par_path: Union[str, Path]) -> Dict[str, np.ndarray]:
    """Read a HITRAN-2004 ``.par`` file: nu0, Sref, g_air, g_self, Elow, n_air, shift
    (float64), mol_id, iso_id (int32), as ``hitran_manager.par_to_dict``."""
    par_path = Path(par_path)
    if not par_path.exists():
        raise FileNotFoundError(f".par file not found: {par_path}")
    data = par_path.read_bytes()
    lib = _lib()
    n = int(lib.lbl_par_count_lines(data, len(data)))
    values = np.zeros((n, 7), dtype=np.float64)
    ids = np.zeros((n, 2), dtype=np.int32)
    status = np.zeros(n, dtype=np.int8)
    if n:
        rc = lib.lbl_par_parse(data, len(data), n, values.ctypes.data, ids.ctypes.data, status.ctypes.data)
        if rc != 0:
            raise RuntimeError("lbl_par_parse: inconsistent line count")
    cols = [ids[:, 0], ids[:, 1]] + [values[:, j] for j in range(7)]
    special = np.flatnonzero((status == PAR_NONASCII) | ((status >= 0) & (status < 9)))
    if special.size == 0:
        keep = status == 9
        out = [c[keep] for c in cols]
    else:
        raw_lines = _split_lines(data)
        fixes = {}
        for i in special.tolist():
            raw = raw_lines[i].decode("utf-8", errors="replace")
            if len(raw) < 155:
                fixes[i] = ([], None, True)
                continue
            vals, exc = _python_fields(raw)
            if exc is not None:
                logger.warning("Malformed line %d in %s: %s", i + 1, par_path.name, exc)
            fixes[i] = (vals, exc, False)
        out = [[] for _ in COLUMNS]
        # ordinary lines go in as blocks between the special ones
        bounds = [-1] + special.tolist() + [n]
        for j in range(len(bounds) - 1):
            lo, hi = bounds[j] + 1, bounds[j + 1]
            if hi > lo:
                keep = status[lo:hi] == 9
                for k in range(9):
                    out[k].append(cols[k][lo:hi][keep])
            if hi < n:
                vals, _, _ = fixes[hi]
                for k, v in enumerate(vals):
                    out[k].append(np.asarray([v], dtype=np.float64 if k >= 2 else np.int32))
        out = [np.concatenate(o) if o else np.zeros(0) for o in out]
    if out[2].size == 0:
        raise HITRANDataError(f"No valid lines read from {par_path}.")
    res = {name: np.asarray(c, dtype=np.int32 if k < 2 else np.float64) for k, (name, c) in
           enumerate(zip(COLUMNS, out))}
    return {k: res[k] for k in ("nu0", "Sref", "g_air", "g_self", "Elow", "n_air", "shift", "mol_id", "iso_id")}


def txt_to_tips(txt_path: Union[str, Path]) -> Tuple[np.ndarray, np.ndarray]:
    """Two-column TIPS table (T, Q); blank and '#' lines ignored (hitran_manager.py:917-963)."""
    txt_path = Path(txt_path)
    if not txt_path.exists():
        raise FileNotFoundError(f"TIPS file not found: {txt_path}")
    t_list, q_list = [], []
    with txt_path.open(encoding="utf-8", errors="replace") as f:
        for raw in f:
            raw = raw.strip()
            if not raw or raw.startswith("#"):
                continue
            parts = raw.split()
            if len(parts) < 2:
                continue
            try:
                t_v, q_v = float(parts[0]), float(parts[1])
            except ValueError:
                continue
            t_list.append(t_v)
            q_list.append(q_v)
    if not t_list:
        raise HITRANDataError(f"No data read from {txt_path}.")
    return np.asarray(t_list, dtype=np.float64), np.asarray(q_list, dtype=np.float64)


def _hapi_molar_mass(mol_name: str, iso: int) -> float:
    """Molar mass from HAPI's isotopologue table (the reference's only source,
    hitran_manager.py:512-552); HAPI is an optional third-party package."""
    try:
        import hapi  # noqa: F401
    except ImportError:
        raise ImportError("\nHAPI (hitran-api) not found in site-packages.\n"
                          "Install it with:  pip install hitran-api\n"
                          "Verify with:      python -m pip show hitran-api") from None
    mol_id = MOLECULE_IDS.get(mol_name)
    record = hapi.ISO.get((mol_id, iso))
    if record is None:
        raise HITRANDataError(f"Isotopologue not found: {mol_name} iso_id={iso}. "
                              "Check list_molecules() for valid IDs.")
    return float(record[3])


def from_files(par_path: Union[str, Path], tips: Dict[tuple, Union[str, Path, Tuple[np.ndarray, np.ndarray]]],
               molar_masses: Optional[Dict[tuple, float]] = None) -> SpectralData:
    """SpectralData from a ``.par`` file and per-isotopologue TIPS (data_loader.py:92-175)."""
    lines = par_to_dict(par_path)
    present = set(zip(lines["mol_id"].tolist(), lines["iso_id"].tolist()))
    missing = present - set(tips.keys())
    if missing:
        raise ValueError(f"Missing TIPS for isotopologue(s): {sorted(missing)}. "
                         "Provide a path or (T, Q) arrays for each (mol_id, iso_id) in the .par file.")
    loaded_tips: Dict[tuple, Tuple[np.ndarray, np.ndarray]] = {}
    for key, val in tips.items():
        if key not in present:
            continue
        if isinstance(val, (str, Path)):
            loaded_tips[key] = txt_to_tips(val)
        else:
            t_arr, q_arr = val
            loaded_tips[key] = (np.asarray(t_arr, dtype=np.float64), np.asarray(q_arr, dtype=np.float64))
    if molar_masses is not None:
        masses = {k: float(v) for k, v in molar_masses.items()}
    else:
        masses = {}
        for mol_id, iso in present:
            mol_name = _ID_TO_MOL.get(mol_id)
            if mol_name is None:
                raise ValueError(f"mol_id={mol_id} not in the internal catalogue. Pass molar_masses manually.")
            masses[(mol_id, iso)] = _hapi_molar_mass(mol_name, iso)
    mol_ids = set(k[0] for k in present)
    molecule = _ID_TO_MOL.get(next(iter(mol_ids))) if len(mol_ids) == 1 else None
    return SpectralData(lines=lines, tips=loaded_tips, molar_masses=masses, molecule=molecule)
