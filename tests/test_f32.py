# SPDX-License-Identifier: 0BSD
"""Plain FP32 field (lpbf_b200_advance_f32) against the FP64 oracle.

Its accuracy target is the FP32 variants' max |T_f32 - T_f64| <= 0.05 K, the
per-step peak trace held to the same bound.  Across temporal depths and task
heights it is bit-identical to itself (one expression per cell), and its
per-step Partials are the exact reduction of its own f32 values: the peak,
the first flat index holding it, and the molten row extent."""
import ctypes

import numpy as np
import pytest

from hedgehog_lpbf_b200 import params as P
from hedgehog_lpbf_b200 import plan as PL
from oracle import oracle as O

pytestmark = pytest.mark.gpu
ATOL_K = 0.05


def _run_f32(k, plan, T0, bc=0, depth=0, rows=0, Tm=1700.0):
    import torch
    from hedgehog_lpbf_b200 import _lib
    L = _lib.lib()
    dev = torch.device("cuda:0")
    n = k.nx * k.ny
    T_a = torch.tensor(np.asarray(T0, dtype=np.float64), device=dev).float()
    T_b = torch.empty_like(T_a)
    s = torch.cuda.current_stream().cuda_stream
    work = torch.empty(L.lpbf_b200_workspace_bytes(), dtype=torch.uint8, device=dev)
    assert L.lpbf_b200_workspace_init(work.data_ptr(), work.numel(), s) == 0
    ring = torch.zeros(24 * len(plan), dtype=torch.uint8, device=dev)
    opts = _lib.Opts(phys=0, bc=bc, T_edge=300.0, Tm=Tm, depth=depth, rows=rows)
    in_b = ctypes.c_int(0)
    st = L.lpbf_b200_advance_f32(T_a.data_ptr(), T_b.data_ptr(), ctypes.byref(k),
                                 plan.ctypes.data, len(plan), ctypes.byref(opts),
                                 ring.data_ptr(), work.data_ptr(), work.numel(), s,
                                 ctypes.byref(in_b))
    assert st == 0, L.lpbf_b200_status_string(st)
    T = T_b if in_b.value else T_a
    torch.cuda.synchronize()
    assert n == T.numel()
    return T.cpu().numpy(), ring.cpu().numpy().view(O.PARTIAL_DTYPE)


def _bench_const(nx, ny):
    mat, pr = P.benchmark_material_process()
    dom = P.Domain(Lx=(nx - 1) * 5e-6, Ly=(ny - 1) * 5e-6, nx=nx, ny=ny)
    return mat, pr, dom, P.make_const(mat, pr, dom, P.dt_fraction(mat, dom))


def _reduce(T, nx, Tm):
    """The Partial of one f32 field, in FP64: peak, first flat index holding
    it, molten rows (T > Tm) min and max (ny and -1 when none)."""
    t = T.astype(np.float64)
    arg = int(np.argmax(t))
    rows = np.nonzero((t.reshape(-1, nx) > Tm).any(axis=1))[0]
    ny = t.size // nx
    return t[arg], arg, (int(rows[0]) if rows.size else ny), (int(rows[-1]) if rows.size else -1)


@pytest.mark.parametrize("bc", [0, 1])
def test_f32_512_2000_steps_within_0p05K(gpu, bc):
    mat, pr, dom, k = _bench_const(512, 512)
    plan = PL.single_track(pr, dom, k.dt, 2000)
    T0 = np.full(512 * 512, 300.0)
    T_ref, ring_ref = O.run(T0, k, PL.laser_array(plan), bc=bc, T_D=300.0, Tm=mat.Tm)
    T, ring = _run_f32(k, plan, T0, bc=bc, Tm=mat.Tm)
    err = float(np.max(np.abs(T.astype(np.float64) - T_ref)))
    perr = float(np.max(np.abs(ring["tmax"] - ring_ref["tmax"])))
    print(f"f32 512^2 x 2000 bc={bc}: max |dT| = {err:.3e} K, peak trace {perr:.3e} K")
    assert err <= ATOL_K
    assert perr <= ATOL_K
    # the last step's Partial is the exact reduction of the returned field
    tm, arg, y0, y1 = _reduce(T, 512, mat.Tm)
    last = ring[-1]
    assert (last["tmax"], last["arg"], last["ymin"], last["ymax"]) == (tm, arg, y0, y1)


def test_f32_depths_bit_identical(gpu):
    mat, pr, dom, k = _bench_const(300, 260)
    rng = np.random.default_rng(9)
    T0 = 300.0 + rng.uniform(0.0, 1500.0, size=300 * 260)
    plan = PL.raster_for_steps(dom, k.dt, 11, V=1.0, hatch=100e-6, n_tracks=2, angle=0.3)
    ref = None
    for depth in (1, 2, 3, 4):
        for rows in (0, 9):
            T, ring = _run_f32(k, plan, T0, depth=depth, rows=rows, Tm=mat.Tm)
            if ref is None:
                ref = (T, ring)
                T_o, _ = O.run(T0, k, PL.laser_array(plan), Tm=mat.Tm)
                assert float(np.max(np.abs(T.astype(np.float64) - T_o))) <= 1e-2
            else:
                assert np.array_equal(T.view(np.uint32), ref[0].view(np.uint32)), (depth, rows)
                assert ring.tobytes() == ref[1].tobytes(), (depth, rows)


@pytest.mark.parametrize("depth", [1, 3])
def test_f32_partials_exact_on_ties_and_unrepresentable_Tm(gpu, depth):
    """A uniform field above Tm with the laser off stays uniform: every cell
    ties for the peak, so each step's Partial must name flat index 0, and
    every row is molten.  Tm = 1609.3 is not an f32 value (the reduction's
    thresholds round it down)."""
    mat, pr, dom, k = _bench_const(264, 200)
    plan = PL.raster_for_steps(dom, k.dt, 6, V=1.0, hatch=100e-6, n_tracks=1)
    plan["q_scale"] = 0.0
    T0 = np.full(264 * 200, 2000.0)
    T, ring = _run_f32(k, plan, T0, depth=depth, Tm=1609.3)
    assert np.all(T == T[0])
    assert np.all(ring["arg"] == 0)
    assert np.all(ring["ymin"] == 0) and np.all(ring["ymax"] == 199)
    assert ring["tmax"][-1] == float(T[0])
    assert np.all(np.diff(ring["tmax"]) < 0)       # cooling, one value per step


def test_f32_rectangular_cells_within_0p05K(gpu):
    """dy != dx: the two-term Laplacian form."""
    mat, pr = P.benchmark_material_process()
    dom = P.Domain(Lx=255 * 5e-6, Ly=199 * 6.5e-6, nx=256, ny=200)
    k = P.make_const(mat, pr, dom, P.dt_fraction(mat, dom))
    assert k.inv_dx2 != k.inv_dy2
    T0 = np.full(256 * 200, 300.0)
    plan = PL.raster_for_steps(dom, k.dt, 400, V=1.0, hatch=100e-6, n_tracks=2, angle=0.5)
    T_ref, ring_ref = O.run(T0, k, PL.laser_array(plan), Tm=mat.Tm)
    T, ring = _run_f32(k, plan, T0, Tm=mat.Tm)
    assert float(np.max(np.abs(T.astype(np.float64) - T_ref))) <= ATOL_K
    assert float(np.max(np.abs(ring["tmax"] - ring_ref["tmax"]))) <= ATOL_K
    tm, arg, y0, y1 = _reduce(T, 256, mat.Tm)
    last = ring[-1]
    assert (last["tmax"], last["arg"], last["ymin"], last["ymax"]) == (tm, arg, y0, y1)


def test_f32_uniform_ambient_field_stays_exact(gpu):
    """No laser, the field at Tamb: the f32 update leaves it exactly at Tamb
    (Laplacian exactly zero, loss below half an ulp)."""
    mat, pr, dom, k = _bench_const(256, 128)
    plan = PL.raster_for_steps(dom, k.dt, 300, V=1.0, hatch=100e-6, n_tracks=1)
    plan["q_scale"] = 0.0
    T, _ = _run_f32(k, plan, np.full(256 * 128, k.Tamb), depth=3, Tm=mat.Tm)
    assert np.all(T == np.float32(k.Tamb))
