"""The C ABI library loads, exports every declared symbol, and the engine fails loudly without CUDA."""

import ctypes
import os
import re

import pytest

from conftest import ROOT
from pylblrtm_b200 import _lib

HEADER = os.path.join(ROOT, "include", "lblgpu.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(lbl_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_bindings_cover_header():
    assert sorted(_lib.SIGNATURES) == declared_functions()


def test_record_sizes_match_header():
    class LayerGroup(ctypes.Structure):
        _fields_ = [(n, ctypes.c_double) for n in ("T", "p_self", "p_air", "col", "q_ratio", "dop")]

    class LineIn(ctypes.Structure):
        _fields_ = [(n, ctypes.c_double) for n in ("nu0", "sref", "g_air", "g_self", "elow", "n_air",
                                                   "shift")] + [("gid", ctypes.c_int), ("src", ctypes.c_int)]

    class LineF32(ctypes.Structure):
        _fields_ = [("nuc", ctypes.c_double), ("j0", ctypes.c_int)] + \
                   [(n, ctypes.c_float) for n in ("b", "a", "y", "amp", "amp_far")]

    assert ctypes.sizeof(LayerGroup) == _lib.SIZEOF_LAYER_GROUP
    assert ctypes.sizeof(LineIn) == _lib.SIZEOF_LINE_IN
    assert ctypes.sizeof(LineF32) == _lib.SIZEOF_LINE_F32
    assert _lib.SIZEOF_LINE_F64 == 4 * 8
    assert ctypes.sizeof(_lib.GemmEpilogue) == _lib.SIZEOF_GEMM_EPILOGUE


def test_surrogate_host_checks():
    lib = _lib.load()
    assert lib.lbl_tensor_map_bytes() == 128
    buf = ctypes.create_string_buffer(128)
    # shape rules are checked before any driver call
    with pytest.raises(RuntimeError, match="multiple of 128"):
        _lib.call("lbl_tensor_map_bf16", ctypes.addressof(buf), 4096, 100, 64, 64)
    ep = _lib.GemmEpilogue(mode=_lib.GEMM_F32)
    with pytest.raises(RuntimeError, match="split-K needs the float32 epilogue"):
        ep2 = _lib.GemmEpilogue(mode=_lib.GEMM_BIAS_GELU)
        _lib.call("lbl_gemm_bf16", ctypes.addressof(buf), ctypes.addressof(buf), 128, 128, 128, 2,
                  ctypes.addressof(ep2), 0, 0)
    with pytest.raises(RuntimeError, match="epilogue buffers"):
        _lib.call("lbl_gemm_bf16", ctypes.addressof(buf), ctypes.addressof(buf), 128, 128, 64, 1,
                  ctypes.addressof(ep), 0, 0)
    with pytest.raises(RuntimeError, match="bad arguments"):
        _lib.call("lbl_adam_step", 0, 0, 0, 0, 1, 0, 1, 1, 1, 1e-3, 0.9, 0.999, 1e-8, 1, 0, 0, 0, 0)


def test_host_queries_and_argument_errors():
    lib = _lib.load()
    assert lib.lbl_abi_version() == 1
    assert lib.lbl_sort_workspace_bytes(10) == 2048 * 12
    assert lib.lbl_sort_workspace_bytes(5000) == 8192 * 12
    # invalid arguments are rejected before any CUDA call
    with pytest.raises(RuntimeError, match="bad arguments"):
        _lib.call("lbl_tau_tiles_f32", 0, 0, 0, 0, 0, 700.0, 0.001, 10, 2000, 25.0, 1, 0, 0, 0, 0)
    with pytest.raises(RuntimeError, match="bad arguments"):
        _lib.call("lbl_faddeeva_f32", 0, 0, 5, 0, 0, 3, 0)
    # Jacobian level-1 workspace: 3 x (16 + 8) coefficients per chunk and row; chunks of at
    # most 1,024 points, so a 2,000-point tile has two and a 5,000-point tile five
    assert lib.lbl_jacobian_ml_work_floats(60, 200001, 2000) == 60 * 101 * 2 * 72
    assert lib.lbl_jacobian_ml_work_floats(2, 10000, 5000) == 2 * 2 * 5 * 72
    assert lib.lbl_jacobian_ml_work_floats(1, 100, 50) == 2 * 72
    assert lib.lbl_jacobian_ml_work_floats(0, 100, 50) == -1
    # forward level-1 workspace: 24 coefficients per (row, chunk); chunks of <= 2048 points
    assert lib.lbl_ml_work_floats(60, 2000, 950) == 60 * 950 * 24
    assert lib.lbl_ml_work_floats(2, 5000, 3) == 2 * 3 * 3 * 24
    assert lib.lbl_ml_work_floats(1, 300, 1) == 24
    assert lib.lbl_ml_work_floats(0, 2000, 1) == -1
    for name in ("lbl_ml_inner_ranges", "lbl_jac_near_ranges"):
        with pytest.raises(RuntimeError, match="bad arguments"):
            _lib.call(name, 0, 0, 700.0, 0.0, 10, 2000, 0.0, 1, 0, 0)
    with pytest.raises(RuntimeError, match="bad arguments"):     # no level-1 workspace
        _lib.call("lbl_jacobian_ml_f32", 1, 1, 10, 1, 0, 0, 1, 60, 60, 700.0, 0.001, 100, 50, 25.0, 0,
                  1, 1, 1, 0, 0, 0, 0, 0)


def test_engine_without_cuda_raises():
    import torch
    if torch.cuda.is_available():
        pytest.skip("CUDA present: the no-GPU error path is exercised on CPU-only hosts")
    import pylblrtm_b200 as lbl
    from pylblrtm_b200 import synthetic
    with pytest.raises(_lib.EngineUnavailable, match="no CUDA device"):
        lbl.compute_transmittance(synthetic.co2_band(50), lbl.us_standard_atmosphere(["CO2"]), 700, 701)


IO_HEADER = os.path.join(ROOT, "include", "lblio.h")


def test_host_library_exports_its_header():
    text = re.sub(r"/\*.*?\*/", "", open(IO_HEADER).read(), flags=re.S)
    names = sorted(set(re.findall(r"\b(lbl_[a-z0-9_]+)\s*\(", text)))
    assert names == sorted(_lib.HOST_SIGNATURES)
    lib = ctypes.CDLL(_lib.IO_LIB_PATH)
    assert all(hasattr(lib, n) for n in names)


def test_line_pairs_scan_rejects_bad_arguments():
    import numpy as np
    host = _lib.load_host()
    pm, pi_, pb = np.zeros(1, np.int32), np.zeros(1, np.int32), np.zeros(1, np.int64)
    n = ctypes.c_int(0)
    smax = ctypes.c_double(0.0)
    mol = np.array([1, 2], np.int32)
    iso = np.array([1, 1], np.int32)
    nu = np.array([700.0, 701.0])
    sh = np.array([0.0, -0.003])
    idx = np.zeros(2, np.int32)
    # two distinct pairs do not fit max_pairs = 1
    assert host.lbl_line_pairs(mol.ctypes.data, iso.ctypes.data, nu.ctypes.data, sh.ctypes.data, 2, 690.0, 710.0,
                               1.0, 1, pm.ctypes.data, pi_.ctypes.data, pb.ctypes.data, ctypes.byref(n),
                               idx.ctypes.data, ctypes.byref(smax)) != 0
    pm, pi_, pb = np.zeros(4, np.int32), np.zeros(4, np.int32), np.zeros(4, np.int64)
    assert host.lbl_line_pairs(mol.ctypes.data, iso.ctypes.data, nu.ctypes.data, sh.ctypes.data, 2, 690.0, 710.0,
                               1.0, 4, pm.ctypes.data, pi_.ctypes.data, pb.ctypes.data, ctypes.byref(n),
                               idx.ctypes.data, ctypes.byref(smax)) == 0
    assert n.value == 2 and list(idx) == [0, 1] and list(pb[:2]) == [1, 1] and smax.value == 0.003


def test_map_index():
    import numpy as np
    host = _lib.load_host()
    idx = np.array([2, 0, 1, 2, 0], np.int32)
    lut = np.array([-1, 5, 7], np.int32)
    out = np.zeros(5, np.int32)
    assert host.lbl_map_index(idx.ctypes.data, 5, lut.ctypes.data, 3, out.ctypes.data) == 0
    assert list(out) == [7, -1, 5, 7, -1]
    bad = np.array([0, 3], np.int32)
    assert host.lbl_map_index(bad.ctypes.data, 2, lut.ctypes.data, 3, out.ctypes.data) != 0
    assert host.lbl_map_index(idx.ctypes.data, 0, None, 0, None) == 0


def _declared_arities(header):
    """Parameter count of every lbl_* function declared in a header."""
    text = re.sub(r"/\*.*?\*/", "", open(header).read(), flags=re.S)
    out = {}
    for m in re.finditer(r"\b(lbl_[a-z0-9_]+)\s*\(([^;{]*?)\)\s*;", text, flags=re.S):
        params = m.group(2).strip()
        out[m.group(1)] = 0 if params in ("", "void") else params.count(",") + 1
    return out


def test_binding_arities_match_headers():
    """Every ctypes binding passes exactly the parameters its C declaration has."""
    for header, sigs in ((HEADER, _lib.SIGNATURES), (IO_HEADER, _lib.HOST_SIGNATURES)):
        arity = _declared_arities(header)
        assert sorted(arity) == sorted(sigs)
        bad = {n: (arity[n], len(sigs[n][1])) for n in sigs if arity[n] != len(sigs[n][1])}
        assert not bad, bad


def test_built_library_is_current():
    """The in-tree libraries are newer than every source they are built from."""
    from pylblrtm_b200.csrc import build as b
    deps = b.SOURCES + b.HEADERS
    assert not b._stale(b.LIB, deps), "liblblgpu.so is older than its sources: rebuild"
    io_deps = ["hitran_par.cpp", "host_scan.cpp", os.path.join("..", "..", "include", "lblio.h")]
    assert not b._stale(b.IO_LIB, io_deps), "liblblio.so is older than its sources: rebuild"
