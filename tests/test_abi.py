# SPDX-License-Identifier: 0BSD
"""The C-ABI library loads and exports every symbol include/*.h declares, and
the headers compile from C and C++ and link against it.  No GPU needed: no
compute entry point is called."""
import ctypes
import os
import re
import subprocess

import pytest

from hedgehog_lpbf_b200 import _lib, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")
DECL = re.compile(r"^\s*(?:void|int|size_t|const\s+char\s*\*)\s*\**\s*(lpbf_\w+)\s*\(", re.M)


def declared_symbols():
    names = set()
    for f in os.listdir(INC):
        if f.endswith((".h", ".hpp")):
            names |= set(DECL.findall(open(os.path.join(INC, f)).read()))
    return sorted(names)


def test_every_declared_symbol_is_bound_and_exported():
    names = declared_symbols()
    assert "lpbf_launch_step" in names and "lpbf_b200_advance" in names
    L = _lib.lib()
    for n in names:
        assert n in _lib.SIGNATURES, f"{n} declared in include/ but not bound in _lib"
        assert hasattr(L, n), f"{n} not exported by {build.LIB}"
    assert set(_lib.SIGNATURES) == set(names)


def test_host_only_entry_points():
    L = _lib.lib()
    assert L.lpbf_b200_version() >= 1
    assert L.lpbf_b200_workspace_bytes() >= 256
    assert L.lpbf_b200_status_string(0) == b"ok"
    o = _lib.Opts(phys=0, bc=0, T_edge=300.0, Tm=1609.0, depth=4, rows=0)
    assert L.lpbf_b200_advance_launches(512, 512, 10, ctypes.byref(o)) == 3
    # argument validation happens before any CUDA call
    assert L.lpbf_b200_advance(None, None, None, None, 0, None, None, None, 0, None, None) == -1


def test_fp32_entry_points_validate_physics_before_any_cuda_call():
    """As lpbf_b200_advance: phys other than 0/1 is an invalid argument, phys 1
    a valid request these entry points do not implement.  The buffers are
    host addresses the calls must not touch (rejected before any launch)."""
    from hedgehog_lpbf_b200.params import StepConst
    L = _lib.lib()
    k = StepConst()
    k.nx, k.ny = 64, 64
    bufs = [ctypes.create_string_buffer(64) for _ in range(4)]
    a = [ctypes.addressof(b) for b in bufs]
    in_b = ctypes.c_int(0)
    for phys, want in ((1, -2), (2, -1), (-1, -1)):
        o = _lib.Opts(phys=phys, bc=0, T_edge=300.0, Tm=1609.0, depth=3, rows=0)
        st = L.lpbf_b200_advance_f32(a[0], a[1], ctypes.byref(k), None, 0, ctypes.byref(o),
                                     None, None, 0, None, ctypes.byref(in_b))
        assert st == want, ("f32", phys, st)
        st = L.lpbf_b200_advance_f32k(a[0], a[1], a[2], a[3], ctypes.byref(k), None, 0,
                                      ctypes.byref(o), None, None, 0, None, ctypes.byref(in_b))
        assert st == want, ("f32k", phys, st)


@pytest.mark.parametrize("lang", ["c", "c++"])
def test_headers_compile_and_link(tmp_path, lang):
    src = tmp_path / ("t.c" if lang == "c" else "t.cpp")
    if lang == "c":
        src.write_text('#include "lpbf_b200.h"\n#include <stdio.h>\n'
                       'int main(void){ printf("%d %zu\\n", lpbf_b200_version(),'
                       ' sizeof(StepConst)); return sizeof(StepConst) != 216; }\n')
        cc = ["gcc", "-std=c11"]
    else:
        src.write_text('#include "lpbf_kernels.hpp"\n#include "lpbf_b200.h"\n#include <cstdio>\n'
                       'int main(){ void (*f)(const double*, double*, const StepConst*, int,'
                       ' cudaStream_t) = lpbf_launch_step; (void)f;'
                       ' std::printf("%d\\n", lpbf_b200_version()); return 0; }\n')
        cc = ["g++", "-std=c++17"]
    exe = tmp_path / "t"
    libdir = os.path.dirname(build.LIB)
    subprocess.run(cc + [str(src), "-I" + INC, "-I/usr/local/cuda/include", "-o", str(exe),
                         "-L" + libdir, "-llpbf_b200", "-Wl,-rpath," + libdir],
                   check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    assert out.split()[0] == "1"


def test_gpu_step_task_header_builds_against_library():
    """include/gpu_step_task.hpp compiles (hh-compat) and links to the library;
    with the reference tree present, so does the reference's own
    hh_gpu_main.cpp against these headers."""
    d = os.path.join(ROOT, "tests", "dropin")
    subprocess.run(["make", "-s", "-C", d, "demo"], check=True)
    assert os.path.exists(os.path.join(ROOT, "tests", "_build", "gpu_task_demo"))
    from oracle import oracle as O
    ref = O.reference_tree()
    if ref and os.path.isdir(os.path.join(ref, "src", "gpu")):
        subprocess.run(["make", "-s", "-C", d, "ref", f"REF={ref}"], check=True)
        assert os.path.exists(os.path.join(ROOT, "tests", "_build", "ref_hhcuda_on_b200"))


def test_manifest_driver_rejects_unusable_manifests(tmp_path):
    """Exit status 4 before any CUDA call, as the reference's manifest mode."""
    d = os.path.join(ROOT, "tests", "dropin")
    subprocess.run(["make", "-s", "-C", d, "demo"], check=True)
    exe = os.path.join(ROOT, "tests", "_build", "manifest_batched")
    r = subprocess.run([exe, f"--manifest={tmp_path / 'nope.csv'}"], capture_output=True, text=True)
    assert r.returncode == 4 and "cannot open manifest" in r.stderr
    bad = tmp_path / "bad.csv"
    bad.write_text("run_id,cond_id,draw_id,config,P_W,V_mps,r0_m,eta,dsub_m,physics\nr,c,d,b,200,1,5e-5,0.4,3e-5,base\n")
    r = subprocess.run([exe, f"--manifest={bad}"], capture_output=True, text=True)
    assert r.returncode == 4 and "missing column 'kmult'" in r.stderr
    empty = tmp_path / "empty.csv"
    empty.write_text("")
    r = subprocess.run([exe, f"--manifest={empty}"], capture_output=True, text=True)
    assert r.returncode == 4
