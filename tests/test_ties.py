# SPDX-License-Identifier: 0BSD
"""Exact ties at the step maximum.  The reference's Partial picks the smallest
flat index among cells at the peak (src/gpu/kernels.cu:205-262); fields with
uniform plateaus hold the peak at many cells at once, spread over strips and
row chunks, so the GPU reductions must keep that rule across tasks, warps,
CTAs and batch scenarios."""
import numpy as np
import pytest

from hedgehog_lpbf_b200 import params as P
from hedgehog_lpbf_b200 import plan as PL
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _const(nx, ny):
    mat, pr = P.benchmark_material_process()
    dom = P.Domain(Lx=(nx - 1) * 5e-6, Ly=(ny - 1) * 5e-6, nx=nx, ny=ny)
    return mat, dom, P.make_const(mat, pr, dom, P.dt_fraction(mat, dom))


def _fields():
    """(name, nx, ny, T0, laser_on)."""
    out = []
    nx, ny = 900, 260
    out.append(("uniform_off", nx, ny, np.full((ny, nx), 300.0), False))
    T = np.full((ny, nx), 300.0)
    T[10:200, 50:700] = 1800.0                       # one plateau over many tasks
    out.append(("plateau", nx, ny, T, False))
    T = np.full((ny, nx), 300.0)
    T[40:70, 20:110] = 1500.0                        # lower rows, first strip
    T[5:35, 300:420] = 1500.0                        # upper rows, later strips
    T[150:180, 700:800] = 1500.0
    out.append(("staircase", nx, ny, T, False))
    T2 = T.copy()
    out.append(("staircase_laser", nx, ny, T2, True))
    return out


def _plan(dom, k, n, on):
    plan = PL.raster_for_steps(dom, k.dt, n, V=1.0, hatch=100e-6, n_tracks=2)
    if not on:
        plan["q_scale"] = 0.0
    return plan


def _check(ring, ring_ref, n):
    assert np.array_equal(ring["arg"][:n], ring_ref["arg"]), (ring["arg"][:n], ring_ref["arg"])
    assert np.array_equal(ring["ymin"][:n], ring_ref["ymin"])
    assert np.array_equal(ring["ymax"][:n], ring_ref["ymax"])
    assert np.max(np.abs(ring["tmax"][:n] - ring_ref["tmax"]) / ring_ref["tmax"]) <= 1e-12


@pytest.mark.parametrize("name,nx,ny,T0,on", _fields(), ids=[f[0] for f in _fields()])
def test_single_field_ties(gpu, name, nx, ny, T0, on):
    from hedgehog_lpbf_b200.solver import Solver, ring_to_numpy
    n = 7
    mat, dom, k = _const(nx, ny)
    plan = _plan(dom, k, n, on)
    _, ring_ref = O.run(T0.ravel(), k, PL.laser_array(plan), Tm=1400.0)
    for depth in (1, 2, 3, 4):
        for rows in (3, 8, 24):
            s = Solver(k, Tm=1400.0, depth=depth, rows=rows, device="cuda:0", T0=T0)
            ring = s.new_ring(n)
            s.advance(plan, ring)
            _check(ring_to_numpy(ring), ring_ref, n)


def test_batch_ties(gpu):
    from hedgehog_lpbf_b200.batch import Batch, Scenario, batch_opts
    n = 7
    scs, refs = [], []
    for name, nx, ny, T0, on in _fields():
        mat, dom, k = _const(nx, ny)
        plan = _plan(dom, k, n, on)
        scs.append(Scenario(k=k, plan=plan, Tm=1400.0, T0=T0))
        refs.append(O.run(T0.ravel(), k, PL.laser_array(plan), Tm=1400.0)[1])
    for depth, rows in ((3, (8, 8, 8, 8)), (2, (3, 3, 3, 3)), (4, (24, 24, 24, 24))):
        b = Batch(scs, n, opts=batch_opts(depth=depth, rows=rows), device="cuda:0")
        b.run(0, n)
        for i in range(len(scs)):
            _check(b.ring(i), refs[i], n)
        b.close()


@pytest.mark.parametrize("bad", [float("nan"), float("inf")])
def test_non_finite_cells_are_flagged_not_trapped(gpu, bad):
    """A NaN or infinite temperature sets bit 1 of the error word; the
    per-step Partials keep the reference rule (NaN never wins, +inf does)."""
    from hedgehog_lpbf_b200.solver import Solver, ring_to_numpy
    n = 5
    mat, dom, k = _const(400, 300)
    plan = _plan(dom, k, n, True)
    T0 = np.full((300, 400), 300.0)
    T0[150, 200] = bad
    s = Solver(k, Tm=1400.0, depth=3, device="cuda:0", T0=T0)
    assert s.read_error() == 0
    ring = s.new_ring(n)
    s.advance(plan, ring)
    assert s.read_error() & 2
    _, ring_ref = O.run(T0.ravel(), k, PL.laser_array(plan), Tm=1400.0)
    r = ring_to_numpy(ring)
    assert np.array_equal(r["arg"], ring_ref["arg"])
    assert np.array_equal(r["tmax"], ring_ref["tmax"]) or np.allclose(
        r["tmax"], ring_ref["tmax"], rtol=1e-12)
    clean = Solver(k, Tm=1400.0, depth=3, device="cuda:0")
    clean.advance(plan, clean.new_ring(n))
    assert clean.read_error() == 0
