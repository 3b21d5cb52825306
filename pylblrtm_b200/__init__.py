"""pylblrtm_b200 — B200-native line-by-line transmittance engine.

Drop-in for the forward path of PyLBLRTM (``pylblrtm/__init__.py:19-72``):
``compute_transmittance``, ``run_forward``, ``load_config``, ``ForwardResult``,
``SpectralData``, ``AtmosphericProfile``, ``us_standard_atmosphere`` and
``list_profile_gases``, ``from_files`` keep the reference's signatures and behaviour; the
line-by-line sums run as hand-written sm_100a CUDA kernels
(``pylblrtm_b200/liblblgpu.so``, C ABI in ``include/lblgpu.h``).
"""

from .atmosphere import AtmosphericProfile
from .batch import transmittance_batch
from .config import ForwardResult, load_config, run_forward
from .forward import compute_transmittance
from .hitran_ids import MOLECULE_IDS
from .hitran_io import HITRANDataError, from_files
from .profiles import list_profile_gases, us_standard_atmosphere
from .spectral_data import SpectralData

__version__ = "0.1.2"

__all__ = [
    "SpectralData",
    "AtmosphericProfile",
    "compute_transmittance",
    "run_forward",
    "load_config",
    "ForwardResult",
    "us_standard_atmosphere",
    "list_profile_gases",
    "MOLECULE_IDS",
    "transmittance_batch",
    "from_files",
    "HITRANDataError",
]
