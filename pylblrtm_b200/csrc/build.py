"""Build liblblgpu.so (sm_100a) in-tree with nvcc.

    python -m pylblrtm_b200.csrc.build          # or pylblrtm_b200.csrc.build.build()

The library lands next to the package (pylblrtm_b200/liblblgpu.so) so that it
travels with the source tree; nothing is installed into site-packages.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
ROOT = os.path.dirname(PKG)
SOURCES = ["capi.cu", "prep.cu", "voigt.cu", "voigt_ml.cu", "voigt_ml_jac.cu", "mlp.cu"]
HEADERS = ["lbl_common.cuh", "faddeeva.cuh", "sum_common.cuh", "weideman_coeffs.h", os.path.join("..", "..", "include", "lblgpu.h")]
LIB = os.path.join(PKG, "liblblgpu.so")
HOST_LIB = os.path.join(PKG, "libfaddeeva_host.so")
IO_LIB = os.path.join(PKG, "liblblio.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build liblblgpu.so")
    return path


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(os.path.join(HERE, d)) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile every .cu source for sm_100a and link liblblgpu.so; returns its path."""
    deps = SOURCES + HEADERS + ["build.py", "faddeeva_host.cpp"]
    if force or _stale(IO_LIB, ["hitran_par.cpp", "host_scan.cpp", os.path.join("..", "..", "include", "lblio.h"),
                                "build.py"]):
        build_io()
    if not force and not _stale(LIB, deps):
        return LIB
    objdir = os.path.join(ROOT, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    for src in SOURCES:
        obj = os.path.join(objdir, src.replace(".cu", ".o"))
        cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "--extended-lambda", "-Xcompiler", "-fPIC",
               "-rdc=false", "-c", os.path.join(HERE, src), "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        subprocess.run(cmd, check=True)
        objs.append(obj)
    tmp = LIB + ".tmp"
    subprocess.run([nvcc(), *ARCH, "-shared", "-o", tmp, *objs, "-lcudart"], check=True)
    os.replace(tmp, LIB)
    build_host_check()
    return LIB


def build_io() -> str:
    """Host (g++) build of the HITRAN reader and line scan, liblblio.so (no CUDA); no
    floating-point contraction, so host arithmetic rounds like NumPy's."""
    tmp = IO_LIB + ".tmp"
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared",
                    os.path.join(HERE, "hitran_par.cpp"), os.path.join(HERE, "host_scan.cpp"), "-o", tmp],
                   check=True)
    os.replace(tmp, IO_LIB)
    return IO_LIB


def build_host_check() -> str:
    """Host (g++) build of faddeeva.cuh used by the CPU accuracy tests."""
    tmp = HOST_LIB + ".tmp"
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared",
                    os.path.join(HERE, "faddeeva_host.cpp"), "-o", tmp], check=True)
    os.replace(tmp, HOST_LIB)
    return HOST_LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
