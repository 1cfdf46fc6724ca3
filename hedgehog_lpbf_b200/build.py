# SPDX-License-Identifier: 0BSD
"""Build recipe of liblpbf_b200.so (sm_100a) -- compiled in-tree with nvcc.

``build()`` recompiles when any source under csrc/ or include/ is newer than
the library.  The library is loaded by ``hedgehog_lpbf_b200._lib`` through
ctypes and by C/C++ callers through include/lpbf_kernels.hpp and
include/lpbf_b200.h.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(PKG, "liblpbf_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
              "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]


def cutlass_include() -> str:
    """CUTLASS/CuTe headers (sm100 UMMA atoms) vendored with the image's
    flashinfer (or tilelang) package; the tensor-core kernels need them."""
    import importlib.util
    for pkg, sub in (("flashinfer", ("data", "cutlass", "include")),
                     ("tilelang", ("3rdparty", "cutlass", "include"))):
        spec = importlib.util.find_spec(pkg)
        if spec is None or not spec.submodule_search_locations:
            continue
        for loc in spec.submodule_search_locations:
            d = os.path.join(loc, *sub)
            if os.path.exists(os.path.join(d, "cute", "atom", "mma_traits_sm100.hpp")):
                return d
    raise RuntimeError("CUTLASS/CuTe headers with sm100 support not found")


def sources() -> list[str]:
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def deps() -> list[str]:
    return (sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.hpp"))
            + glob.glob(os.path.join(INCLUDE, "*.h*")))


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found: liblpbf_b200.so cannot be built")
    return cand


def stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(d) > t for d in deps())


def build(force: bool = False, verbose: bool = False, jobs: int | None = None) -> str:
    if not force and not stale():
        return LIB
    objdir = os.path.join(PKG, "_build")
    os.makedirs(objdir, exist_ok=True)
    inc = ["-I" + INCLUDE, "-I" + CSRC, "-I" + cutlass_include()]
    objs, procs = [], []
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        cmd = [nvcc(), *ARCH, *NVCC_FLAGS, *inc, "-c", src, "-o", obj]
        if verbose:
            cmd += ["-Xptxas", "-v"]
            print(" ".join(cmd), file=sys.stderr)
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
        objs.append(obj)
    failed = []
    for src, pr in procs:
        out, _ = pr.communicate()
        if verbose or pr.returncode != 0:
            sys.stderr.write(out.decode())
        if pr.returncode != 0:
            failed.append(src)
    if failed:
        raise RuntimeError("nvcc failed on " + ", ".join(failed))
    tmp = LIB + ".tmp"
    subprocess.run([nvcc(), *ARCH, "-shared", "-Xcompiler", "-fPIC", *objs, "-o", tmp,
                    "-lcudart"], check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
