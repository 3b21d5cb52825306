"""ctypes binding of liblblgpu.so (the sm_100a kernels behind include/lblgpu.h).

The library is built in-tree (``pylblrtm_b200/liblblgpu.so``) by
``pylblrtm_b200.csrc.build``. There is no CPU implementation of the engine:
if the library or a CUDA device is missing, every engine call raises.
"""

from __future__ import annotations

import ctypes
import os
import threading

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "liblblgpu.so")

LBL_OK = 0
LBL_DETERMINISTIC = 1    # flag of the multi-level summation and Jacobian kernels

# byte sizes of the records declared in include/lblgpu.h
SIZEOF_LAYER_GROUP = 48
SIZEOF_LINE_IN = 64
SIZEOF_LINE_F64 = 32
SIZEOF_LINE_F32 = 32
SIZEOF_LINE_JAC = 32

_P = ctypes.c_void_p
_I = ctypes.c_int
_L = ctypes.c_longlong
_D = ctypes.c_double
_S = ctypes.c_size_t
_F = ctypes.c_float

# name -> (restype, argtypes); every function of include/lblgpu.h
SIGNATURES = {
    "lbl_last_error": (ctypes.c_char_p, []),
    "lbl_abi_version": (_I, []),
    "lbl_build_layers": (_I, [_P, _P, _P, _I, _I, _I, _D, _P, _P, _P, _P, _P]),
    "lbl_layer_groups": (_I, [_P, _P, _P, _P, _I, _I, _I, _I, _P, _P, _P, _P, _P, _P, _P, _P]),
    "lbl_sort_workspace_bytes": (_S, [_I]),
    "lbl_sort_lines": (_I, [_P, _P, _P, _I, _D, _D, _D, _P, _S, _P, _P, _P, _P]),
    "lbl_sort_lines_noalloc": (_I, [_P, _P, _P, _I, _D, _D, _D, _P, _P, _P, _P]),
    "lbl_gather_lines": (_I, [_P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _I, _P, _P]),
    "lbl_tile_ranges": (_I, [_P, _P, _D, _D, _L, _I, _D, _D, _I, _P, _P]),
    "lbl_line_prep_f64": (_I, [_P, _P, _I, _P, _I, _I, _P, _P, _P]),
    "lbl_line_prep_f32": (_I, [_P, _P, _I, _P, _I, _I, _D, _D, _P, _P, _P]),
    "lbl_tau_tiles_f64": (_I, [_P, _I, _P, _P, _I, _D, _D, _L, _I, _D, _I, _P, _P, _P, _P]),
    "lbl_tau_tiles_f32": (_I, [_P, _I, _P, _P, _I, _D, _D, _L, _I, _D, _I, _P, _P, _P, _P]),
    "lbl_ml_inner_ranges": (_I, [_P, _P, _D, _D, _L, _I, _D, _I, _P, _P]),
    "lbl_tau_tiles_ml_f32": (_I, [_P, _I, _P, _P, _P, _P, _I, _D, _D, _L, _I, _D, _I, _P, _P, _P, _P, _I, _I, _I,
                                  _P]),
    "lbl_ml_work_floats": (_L, [_I, _I, _I]),
    "lbl_line_prep_jac": (_I, [_P, _I, _P, _I, _I, _P, _P, _P, _P, _I, _P, _P, _P]),
    "lbl_jacobian_ml_f32": (_I, [_P, _P, _I, _P, _P, _P, _P, _I, _I, _D, _D, _L, _I, _D, _P, _P, _P, _P, _P, _P,
                                 _P, _I, _P]),
    "lbl_jac_near_ranges": (_I, [_P, _P, _D, _D, _L, _I, _D, _I, _P, _P]),
    "lbl_jacobian_ml_work_floats": (_L, [_I, _L, _I]),
    "lbl_layer_sum_exp_f32": (_I, [_P, _I, _I, _L, _P, _P, _P, _P]),
    "lbl_layer_sum_exp_f64": (_I, [_P, _I, _I, _L, _P, _P, _P, _P]),
    "lbl_channel_mean_f32": (_I, [_P, _I, _I, _L, _P, _L, _I, _I, _P, _P]),
    "lbl_channel_mean_f64": (_I, [_P, _I, _I, _L, _P, _L, _I, _I, _P, _P]),
    "lbl_faddeeva_f64": (_I, [_P, _P, _L, _P, _P, _P]),
    "lbl_faddeeva_f32": (_I, [_P, _P, _L, _P, _P, _I, _P]),
    "lbl_probe_fma_f32": (_I, [_P, _I, _I, _P]),
    "lbl_tensor_map_bytes": (_S, []),
    "lbl_tensor_map_bf16": (_I, [_P, _P, _L, _L, _L]),
    "lbl_gemm_bf16": (_I, [_P, _P, _I, _I, _I, _I, _P, _P, _P]),
    "lbl_adam_step": (_I, [_P, _P, _P, _P, _I, _L, _I, _I, _I, _F, _F, _F, _F, _I, _P, _P, _I, _P]),
    "lbl_rowsum_bf16": (_I, [_P, _I, _I, _I, _P, _P]),
    "lbl_pack_inputs_bf16": (_I, [_P, _I, _I, _P, _P, _P, _I, _P, _I, _P]),
    "lbl_ensemble_gate": (_I, [_P, _I, _L, _I, _I, _I, _P, _F, _F, _P, _P, _P, _P]),
}

# epilogue modes of lbl_gemm_bf16
GEMM_F32, GEMM_BIAS_GELU, GEMM_BIAS_SIGMOID, GEMM_DGELU = 0, 1, 2, 3


class GemmEpilogue(ctypes.Structure):
    """LblGemmEpilogue of include/lblgpu.h (136 bytes)."""
    _fields_ = [("mode", _I), ("n_valid", _I), ("bias", _P), ("out_f32", _P), ("ld_f32", _L),
                ("split_stride", _L), ("z_out", _P), ("ld_z", _L), ("z_in", _P), ("ld_zin", _L),
                ("y", _P), ("ld_y", _L), ("y_t", _P), ("ld_yt", _L), ("target", _P), ("ld_target", _L),
                ("grad_scale", ctypes.c_float), ("pad0", _I), ("loss", _P)]


SIZEOF_GEMM_EPILOGUE = 136

# host-side helpers (liblblio.so, include/lblio.h): no CUDA
IO_LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "liblblio.so")
HOST_SIGNATURES = {
    "lbl_par_count_lines": (_L, [ctypes.c_char_p, _L]),
    "lbl_par_parse": (_I, [ctypes.c_char_p, _L, _L, _P, _P, _P]),
    "lbl_line_pairs": (_I, [_P, _P, _P, _P, _L, _D, _D, _D, _I, _P, _P, _P, _P, _P, _P]),
    "lbl_map_index": (_I, [_P, _L, _P, _I, _P]),
    "lbl_count_band": (_L, [_P, _P, _P, _L, _D, _D, _D]),
}

_lock = threading.Lock()
_lib = None
_host = None


def load_host() -> ctypes.CDLL:
    """Load liblblio.so (host helpers) once and declare its signatures."""
    global _host
    with _lock:
        if _host is None:
            if not os.path.exists(IO_LIB_PATH):
                raise EngineUnavailable(f"{IO_LIB_PATH} is missing; build it with "
                                        "`python -m pylblrtm_b200.csrc.build`")
            lib = ctypes.CDLL(IO_LIB_PATH)
            for name, (res, args) in HOST_SIGNATURES.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _host = lib
    return _host


class EngineUnavailable(RuntimeError):
    """The CUDA library or a CUDA device is missing (there is no CPU fallback)."""


def load() -> ctypes.CDLL:
    """Load liblblgpu.so once and declare every signature."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise EngineUnavailable(
                    f"{LIB_PATH} is missing; build it with `python -m pylblrtm_b200.csrc.build` "
                    "(the line-by-line engine has no CPU implementation)")
            lib = ctypes.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _lib = lib
    return _lib


def call(name: str, *args) -> None:
    """Call an entry point and raise RuntimeError with the library's message on failure."""
    lib = load()
    status = getattr(lib, name)(*args)
    if status != LBL_OK:
        msg = lib.lbl_last_error().decode(errors="replace")
        raise RuntimeError(f"{name} failed (status {status}): {msg}")


def ptr(t) -> int:
    """Device address of a torch tensor (or 0 for None)."""
    return 0 if t is None else t.data_ptr()
