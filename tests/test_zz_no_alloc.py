# SPDX-License-Identifier: 0BSD
"""The no-allocation entry point, lpbf_b200_advance_noalloc.

It exists for callers that cannot allocate device memory (a task graph whose
device memory is fixed at start-up, cgo/JNI bindings that only hand raw
device pointers through, hosts where a cudaMalloc would synchronize the
device at a forbidden point): it takes no workspace and keeps its scratch in
a fixed array inside the library.  This file checks, through the C-ABI, that
two calls in a row give the same fields and per-step Partials as the
workspace entry point, lpbf_b200_advance, within the parity tolerance used
throughout (max relative error 1e-12 on the field, exact Partials), and that
it rejects what it does not support.  It is named to be collected last.
"""
import ctypes

import numpy as np
import pytest

from hedgehog_lpbf_b200 import params as P
from hedgehog_lpbf_b200 import plan as PL

pytestmark = pytest.mark.gpu
RTOL = 1e-12


def _rel_err(a, b):
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1.0)))


def _advance(L, torch, k, plan, T0, opts, noalloc, work=None):
    dev = torch.device("cuda:0")
    a = torch.tensor(T0, device=dev)
    b = torch.empty_like(a)
    n = len(plan)
    ring = torch.zeros(24 * n, dtype=torch.uint8, device=dev)
    in_b = ctypes.c_int(-1)
    stream = torch.cuda.current_stream().cuda_stream
    if noalloc:
        st = L.lpbf_b200_advance_noalloc(a.data_ptr(), b.data_ptr(), ctypes.byref(k),
                                         plan.ctypes.data, n, ctypes.byref(opts),
                                         ring.data_ptr(), stream, ctypes.byref(in_b))
    else:
        st = L.lpbf_b200_advance(a.data_ptr(), b.data_ptr(), ctypes.byref(k), plan.ctypes.data,
                                 n, ctypes.byref(opts), ring.data_ptr(), work.data_ptr(),
                                 work.numel(), stream, ctypes.byref(in_b))
    assert st == 0, L.lpbf_b200_status_string(st)
    torch.cuda.synchronize()
    T = (b if in_b.value else a).cpu().numpy()
    return T, ring.cpu().numpy()


@pytest.mark.parametrize("depth", [3, 4])
def test_no_alloc_matches_workspace_entry_point_twice(gpu, depth):
    import torch
    from hedgehog_lpbf_b200 import _lib
    L = _lib.lib()
    mat, pr = P.benchmark_material_process()
    dom = P.Domain(Lx=511 * 5e-6, Ly=383 * 5e-6, nx=512, ny=384)
    k = P.make_const(mat, pr, dom, P.dt_fraction(mat, dom))
    opts = _lib.Opts(phys=0, bc=0, T_edge=300.0, Tm=mat.Tm, depth=depth, rows=0)
    work = torch.empty(L.lpbf_b200_workspace_bytes(), dtype=torch.uint8, device="cuda:0")
    assert L.lpbf_b200_workspace_init(work.data_ptr(), work.numel(),
                                      torch.cuda.current_stream().cuda_stream) == 0
    rng = np.random.default_rng(depth)
    cases = [
        (np.full(512 * 384, 300.0), PL.single_track(pr, dom, k.dt, 37)),
        (300.0 + rng.uniform(0.0, 2000.0, 512 * 384),
         PL.raster_for_steps(dom, k.dt, 29, V=1.0, hatch=100e-6, n_tracks=2, angle=0.4)),
    ]
    for T0, plan in cases:                     # two calls in a row
        T_ref, r_ref = _advance(L, torch, k, plan, T0, opts, noalloc=False, work=work)
        T_na, r_na = _advance(L, torch, k, plan, T0, opts, noalloc=True)
        assert _rel_err(T_na, T_ref) <= RTOL
        assert r_na.tobytes() == r_ref.tobytes()


def test_no_alloc_rejects_extended_physics(gpu):
    import torch
    from hedgehog_lpbf_b200 import _lib
    L = _lib.lib()
    mat, pr = P.benchmark_material_process()
    dom = P.square_domain(64)
    k = P.make_const(mat, pr, dom, P.dt_fraction(mat, dom))
    opts = _lib.Opts(phys=1, bc=0, T_edge=300.0, Tm=mat.Tm, depth=1, rows=0)
    a = torch.full((64, 64), 300.0, dtype=torch.float64, device="cuda:0")
    b = torch.empty_like(a)
    plan = PL.single_track(pr, dom, k.dt, 2)
    in_b = ctypes.c_int(0)
    st = L.lpbf_b200_advance_noalloc(a.data_ptr(), b.data_ptr(), ctypes.byref(k),
                                     plan.ctypes.data, 2, ctypes.byref(opts), None,
                                     torch.cuda.current_stream().cuda_stream, ctypes.byref(in_b))
    assert st == -2
