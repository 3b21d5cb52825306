"""Line-parameter container (drop-in for ``pylblrtm/spectral_data.py:14-78``).

The forward engine reads ``lines`` (nine arrays), ``tips`` and
``molar_masses`` from this object and uploads them to the device on each call;
the host-side ``Q`` method stays for API compatibility, while the engine
interpolates the same tables on the GPU (``csrc/prep.cu``).
"""

from dataclasses import dataclass
from typing import Dict, Optional, Tuple

import numpy as np

LINE_KEYS = ("nu0", "Sref", "g_air", "g_self", "Elow", "n_air", "shift", "mol_id", "iso_id")


@dataclass
class SpectralData:
    """Line parameters, partition-sum tables and molar masses.

    ``lines`` maps the keys ``nu0, Sref, g_air, g_self, Elow, n_air, shift,
    mol_id, iso_id`` to equal-length 1-D arrays. ``tips`` maps
    ``(mol_id, iso_id)`` to a ``(T, Q)`` pair of 1-D arrays (T increasing);
    ``molar_masses`` maps the same keys to g/mol.
    """

    lines: Dict[str, np.ndarray]
    tips: Dict[tuple, Tuple[np.ndarray, np.ndarray]]
    molar_masses: Dict[tuple, float]
    molecule: Optional[str] = None

    def Q(self, T: float, mol_id: int, iso_id: int) -> float:
        """Partition sum at ``T`` by linear interpolation, clamped at the table
        ends (``pylblrtm/spectral_data.py:43-52``)."""
        key = (int(mol_id), int(iso_id))
        if key not in self.tips:
            raise KeyError(
                f"No TIPS data for (mol_id={mol_id}, iso_id={iso_id}). "
                f"Available: {sorted(self.tips.keys())}"
            )
        t_arr, q_arr = self.tips[key]
        return float(np.interp(T, t_arr, q_arr))

    @property
    def nu0(self) -> np.ndarray:
        return self.lines["nu0"]

    @property
    def Sref(self) -> np.ndarray:
        return self.lines["Sref"]

    @property
    def n_lines(self) -> int:
        return len(self.lines["nu0"])

    def __repr__(self) -> str:
        keys = sorted(self.tips.keys())
        nu = self.lines["nu0"]
        isos = ", ".join(f"({m},{i})" for m, i in keys)
        label = self.molecule or "multi-molecule"
        return (
            f"SpectralData({label}, (mol_id,iso_id)=[{isos}], {self.n_lines} lines, "
            f"nu=[{nu.min():.1f}, {nu.max():.1f}] cm-1)"
        )
