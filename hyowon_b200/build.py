"""Build the in-tree native library hyowon_b200/libhyowon_pm.so for sm_100a.

Every translation unit is compiled by nvcc with
``-gencode arch=compute_100a,code=sm_100a -lineinfo``. The binary64 kernels are
compiled with ``--fmad=false`` so that no multiply-add is contracted, matching
the reference's ``-ffp-contract=off`` build (bit-parity of cell assignment,
CIC weights, gradient stencil and KDK arithmetic). The precision form keeps
FMA contraction.

    python -m hyowon_b200.build
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libhyowon_pm.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
          "-I", os.path.join(ROOT, "include"), "-I", CSRC, "--expt-relaxed-constexpr"]
# Extra nvcc flags for every unit, e.g. HYOWON_NVCC_DEFS="-DHYOWON_KICK32_MINB=4" to
# build a tuning variant (pass --force: the object files do not track flags).
COMMON += os.environ.get("HYOWON_NVCC_DEFS", "").split()

# (source, extra flags)
UNITS = [
    ("pm_fp64.cu", ["--fmad=false"]),
    ("pm_sort.cu", []),
    ("pm_lpt.cu", []),
    ("pm_adjoint.cu", []),
    ("pm_tree.cu", []),
    ("pm_handle.cu", ["--fmad=false"]),
    ("pm_fp32.cu", []),
    ("pm_poisson.cu", []),
    ("pm_noalloc.cu", ["--fmad=false"]),
    ("pm_diag.cu", ["--fmad=false"]),
    ("pm_pk.cu", ["--fmad=false"]),
    ("pm_ic.cu", ["--fmad=false"]),
    ("pm_snapshot.cu", ["--fmad=false"]),
    ("cosmology.cpp", []),
]


def _needs(obj: str, deps: list[str]) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers += [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include"))]
    objs = []
    for src, extra in UNITS:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _needs(o, [s, __file__] + headers):
            cmd = [NVCC] + ARCH + COMMON + extra + ["-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
    if force or _needs(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + [
            "-cudart", "static", "-lcufft", "-Xlinker", "-rpath,/usr/local/cuda/lib64"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
