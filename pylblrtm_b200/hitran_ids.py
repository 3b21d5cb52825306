"""HITRAN molecule numbering used to map line ``mol_id`` values to gas names.

The numbering is HITRAN's own global molecule index; it has to be identical to
the table the reference forward model uses (``pylblrtm/hitran_manager.py:89-101``)
so that ``mol_id`` → gas-name resolution, and therefore which lines are skipped
with a warning, is the same in both.
"""

from typing import Dict

MOLECULE_IDS: Dict[str, int] = {
    "H2O": 1, "CO2": 2, "O3": 3, "N2O": 4, "CO": 5, "CH4": 6, "O2": 7,
    "NO": 8, "SO2": 9, "NO2": 10, "NH3": 11, "HNO3": 12, "OH": 13, "HF": 14,
    "HCl": 15, "HBr": 16, "HI": 17, "ClO": 18, "OCS": 19, "H2CO": 20,
    "HOCl": 21, "N2": 22, "HCN": 23, "CH3Cl": 24, "H2O2": 25, "C2H2": 26,
    "C2H6": 27, "PH3": 28, "COF2": 29, "SF6": 30, "H2S": 31, "HCOOH": 32,
    "HO2": 33, "O": 34, "ClONO2": 35, "NO+": 36, "HOBr": 37, "C2H4": 38,
    "CH3OH": 39, "CH3Br": 40, "CH3CN": 41, "CF4": 42, "C4H2": 43, "HC3N": 44,
    "H2": 45, "CS": 46, "SO3": 47, "C2N2": 48, "COCl2": 49, "SO": 51,
    "CH3F": 52, "GeH4": 53, "CS2": 54, "CH3I": 55, "NF3": 56,
}

MOL_ID_TO_NAME: Dict[int, str] = {v: k for k, v in MOLECULE_IDS.items()}
