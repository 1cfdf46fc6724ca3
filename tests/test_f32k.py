# SPDX-License-Identifier: 0BSD
"""FP32 compensated variant (lpbf_b200_advance_f32k) against the FP64 oracle.

Its accuracy target is max |T_f32k - T_f64| <= 0.05 K; the per-step peak
trace is held to the same absolute bound.  Across temporal depths and chunk
sizes the variant is bit-identical to itself (one expression per cell)."""
import ctypes

import numpy as np
import pytest

from hedgehog_lpbf_b200 import params as P
from hedgehog_lpbf_b200 import plan as PL
from oracle import oracle as O

pytestmark = pytest.mark.gpu
ATOL_K = 0.05


def _run_f32k(k, plan, T0, bc=0, depth=0, rows=0, Tm=1700.0):
    import torch
    from hedgehog_lpbf_b200 import _lib
    L = _lib.lib()
    dev = torch.device("cuda:0")
    n = k.nx * k.ny
    T = torch.tensor(np.asarray(T0, dtype=np.float64), device=dev)
    hi_a = torch.empty(n, dtype=torch.float32, device=dev)
    lo_a = torch.empty_like(hi_a)
    hi_b = torch.empty_like(hi_a)
    lo_b = torch.empty_like(hi_a)
    s = torch.cuda.current_stream().cuda_stream
    assert L.lpbf_b200_f32k_split(T.data_ptr(), hi_a.data_ptr(), lo_a.data_ptr(), n, s) == 0
    work = torch.empty(L.lpbf_b200_workspace_bytes(), dtype=torch.uint8, device=dev)
    assert L.lpbf_b200_workspace_init(work.data_ptr(), work.numel(), s) == 0
    ring = torch.zeros(24 * len(plan), dtype=torch.uint8, device=dev)
    opts = _lib.Opts(phys=0, bc=bc, T_edge=300.0, Tm=Tm, depth=depth, rows=rows)
    in_b = ctypes.c_int(0)
    st = L.lpbf_b200_advance_f32k(hi_a.data_ptr(), lo_a.data_ptr(), hi_b.data_ptr(),
                                  lo_b.data_ptr(), ctypes.byref(k), plan.ctypes.data, len(plan),
                                  ctypes.byref(opts), ring.data_ptr(), work.data_ptr(),
                                  work.numel(), s, ctypes.byref(in_b))
    assert st == 0, L.lpbf_b200_status_string(st)
    hi, lo = (hi_b, lo_b) if in_b.value else (hi_a, lo_a)
    out = torch.empty(n, dtype=torch.float64, device=dev)
    assert L.lpbf_b200_f32k_join(hi.data_ptr(), lo.data_ptr(), out.data_ptr(), n, s) == 0
    torch.cuda.synchronize()
    return out.cpu().numpy(), ring.cpu().numpy().view(O.PARTIAL_DTYPE), hi.cpu().numpy()


def _bench_const(nx, ny):
    mat, pr = P.benchmark_material_process()
    dom = P.Domain(Lx=(nx - 1) * 5e-6, Ly=(ny - 1) * 5e-6, nx=nx, ny=ny)
    return mat, pr, dom, P.make_const(mat, pr, dom, P.dt_fraction(mat, dom))


@pytest.mark.parametrize("bc", [0, 1])
def test_f32k_512_2000_steps_within_0p05K(gpu, bc):
    mat, pr, dom, k = _bench_const(512, 512)
    plan = PL.single_track(pr, dom, k.dt, 2000)
    T0 = np.full(512 * 512, 300.0)
    T_ref, ring_ref = O.run(T0, k, PL.laser_array(plan), bc=bc, T_D=300.0, Tm=mat.Tm)
    T, ring, _ = _run_f32k(k, plan, T0, bc=bc, Tm=mat.Tm)
    err = float(np.max(np.abs(T - T_ref)))
    print(f"f32k 512^2 x 2000 bc={bc}: max |dT| = {err:.3e} K")
    assert err <= ATOL_K
    assert float(np.max(np.abs(ring["tmax"] - ring_ref["tmax"]))) <= ATOL_K


def test_f32k_depths_bit_identical(gpu):
    mat, pr, dom, k = _bench_const(300, 260)
    rng = np.random.default_rng(9)
    T0 = 300.0 + rng.uniform(0.0, 1500.0, size=300 * 260)
    plan = PL.raster_for_steps(dom, k.dt, 11, V=1.0, hatch=100e-6, n_tracks=2, angle=0.3)
    ref = None
    for depth in (1, 2, 3, 4):
        for rows in (0, 9):
            T, ring, hi = _run_f32k(k, plan, T0, depth=depth, rows=rows, Tm=mat.Tm)
            if ref is None:
                ref = (T, ring)
                T_o, _ = O.run(T0, k, PL.laser_array(plan), Tm=mat.Tm)
                assert float(np.max(np.abs(T - T_o))) <= 1e-3
            else:
                assert np.array_equal(T.view(np.uint64), ref[0].view(np.uint64)), (depth, rows)
                assert ring.tobytes() == ref[1].tobytes(), (depth, rows)


def test_f32k_split_join_round_trip(gpu):
    import torch
    from hedgehog_lpbf_b200 import _lib
    L = _lib.lib()
    rng = np.random.default_rng(2)
    x = 300.0 + rng.uniform(0, 5000, 10007)
    d = torch.tensor(x, device="cuda:0")
    hi = torch.empty(x.size, dtype=torch.float32, device="cuda:0")
    lo = torch.empty_like(hi)
    out = torch.empty_like(d)
    s = torch.cuda.current_stream().cuda_stream
    assert L.lpbf_b200_f32k_split(d.data_ptr(), hi.data_ptr(), lo.data_ptr(), x.size, s) == 0
    assert L.lpbf_b200_f32k_join(hi.data_ptr(), lo.data_ptr(), out.data_ptr(), x.size, s) == 0
    torch.cuda.synchronize()
    y = out.cpu().numpy()
    assert np.max(np.abs(y - x) / x) < 2.0 ** -46     # two f32 halves keep ~48 bits


def test_f32k_substrate_temperature_differs_from_ambient(gpu):
    mat, pr = P.benchmark_material_process()
    pr.Tsub = 420.0
    dom = P.Domain(Lx=299 * 5e-6, Ly=259 * 5e-6, nx=300, ny=260)
    k = P.make_const(mat, pr, dom, P.dt_fraction(mat, dom))
    T0 = np.full(300 * 260, 300.0)
    plan = PL.raster_for_steps(dom, k.dt, 400, V=1.0, hatch=100e-6, n_tracks=2)
    T_ref, ring_ref = O.run(T0, k, PL.laser_array(plan), Tm=mat.Tm)
    T, ring, _ = _run_f32k(k, plan, T0, Tm=mat.Tm)
    assert float(np.max(np.abs(T - T_ref))) <= ATOL_K
    assert float(np.max(np.abs(ring["tmax"] - ring_ref["tmax"]))) <= ATOL_K


def test_f32k_rectangular_cells_within_0p05K(gpu):
    """dy != dx: the two-term Laplacian form of the compensated update."""
    mat, pr = P.benchmark_material_process()
    dom = P.Domain(Lx=255 * 5e-6, Ly=199 * 6.5e-6, nx=256, ny=200)
    k = P.make_const(mat, pr, dom, P.dt_fraction(mat, dom))
    assert k.inv_dx2 != k.inv_dy2
    T0 = np.full(256 * 200, 300.0)
    plan = PL.raster_for_steps(dom, k.dt, 400, V=1.0, hatch=100e-6, n_tracks=2, angle=0.5)
    T_ref, ring_ref = O.run(T0, k, PL.laser_array(plan), Tm=mat.Tm)
    T, ring, _ = _run_f32k(k, plan, T0, Tm=mat.Tm)
    assert float(np.max(np.abs(T - T_ref))) <= ATOL_K
    assert float(np.max(np.abs(ring["tmax"] - ring_ref["tmax"]))) <= ATOL_K
