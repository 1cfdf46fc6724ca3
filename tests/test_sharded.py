# SPDX-License-Identifier: 0BSD
"""Row-strip sharding of one field (hedgehog_lpbf_b200.sharded).

CPU: the strip layout, the combination of strip Partials, and the halo
exchange with the oracle advancing each strip (strips in one process, and
two gloo ranks on 127.0.0.1), against the oracle's whole-field run.
GPU: strips advanced by lpbf_b200_advance_rows equal the single-field
solver bit for bit (fields and per-step Partials)."""
import os
import socket

import numpy as np
import pytest
import torch

from hedgehog_lpbf_b200 import params as P
from hedgehog_lpbf_b200 import plan as PL
from hedgehog_lpbf_b200 import sharded as S
from hedgehog_lpbf_b200.solver import PARTIAL_DTYPE

RTOL = 1e-12


def _const(nx, ny):
    mat, pr = P.benchmark_material_process()
    dom = P.Domain(Lx=(nx - 1) * 5e-6, Ly=(ny - 1) * 5e-6, nx=nx, ny=ny)
    return mat, dom, P.make_const(mat, pr, dom, P.dt_fraction(mat, dom))


def _case(nx=96, ny=70, n=11, seed=4):
    mat, dom, k = _const(nx, ny)
    rng = np.random.default_rng(seed)
    T0 = 300.0 + rng.uniform(0.0, 1500.0, size=(ny, nx))
    # the spot crosses every strip boundary; off for a few steps (cooling)
    las = np.stack([np.linspace(0.2, 0.8, n) * dom.Lx, np.linspace(0.05, 0.95, n) * dom.Ly,
                    (np.arange(n) % 5 != 4).astype(float)], axis=1)
    plan = np.zeros(n, dtype=PL.TICK_DTYPE)
    plan["step"] = np.arange(n)
    plan["x_l"], plan["y_l"], plan["q_scale"] = las[:, 0], las[:, 1], las[:, 2]
    return mat, k, T0, las, plan


class OracleStripStepper:
    """The oracle advancing one strip buffer step by step (the laser's y
    taken relative to the buffer's first row), with the Partial of the
    owned rows in the field's numbering."""

    def __init__(self, bc=0, T_edge=300.0, Tm=1609.0):
        self.bc, self.T_edge, self.Tm = bc, T_edge, Tm

    def __call__(self, T_in, T_out, ks, gny, strip, plan, ring):
        from oracle import oracle as O
        nx, rows = ks.nx, ks.ny
        T = T_in.numpy().copy().ravel()
        parts = np.zeros(len(plan), dtype=PARTIAL_DTYPE)
        kk = type(ks).from_buffer_copy(bytes(ks))
        for t in range(len(plan)):
            kk.x_l = plan["x_l"][t]
            kk.y_l = plan["y_l"][t] - strip.row0 * ks.dy
            kk.q_scale = plan["q_scale"][t]
            T = O.step(T, kk, 0, self.bc, self.T_edge)
            own = T.reshape(rows, nx)[strip.lo:strip.hi]
            tm, ag, mn, mx = O.reduce(own.ravel(), nx, strip.hi - strip.lo, self.Tm)
            first = strip.row0 + strip.lo
            neutral = ag >= nx * (strip.hi - strip.lo)
            parts[t] = (tm, nx * gny if neutral else ag + first * nx,
                        gny if mx < 0 else mn + first, -1 if mx < 0 else mx + first)
        T_out[strip.lo:strip.hi] = torch.as_tensor(T.reshape(rows, nx)[strip.lo:strip.hi])
        if ring is not None:
            ring.copy_(torch.as_tensor(parts.view(np.uint8)))


def _check(T, parts, T_ref, ring_ref):
    err = np.max(np.abs(T - T_ref) / np.maximum(np.abs(T_ref), 1.0))
    assert err <= RTOL, err
    assert np.max(np.abs(parts["tmax"] - ring_ref["tmax"]) / ring_ref["tmax"]) <= RTOL
    assert np.array_equal(parts["ymin"], ring_ref["ymin"])
    assert np.array_equal(parts["ymax"], ring_ref["ymax"])


# ---- layout and combination ---------------------------------------------------

@pytest.mark.parametrize("ny,parts,halo", [(70, 3, 3), (9, 3, 3), (100, 7, 4), (5, 1, 4)])
def test_strip_layout_covers_the_field(ny, parts, halo):
    lay = S.strip_layout(ny, parts, halo)
    assert [s.a for s in lay][0] == 0 and lay[-1].b == ny
    assert all(lay[i].b == lay[i + 1].a for i in range(parts - 1))
    assert max(s.b - s.a for s in lay) - min(s.b - s.a for s in lay) <= 1
    assert lay[0].top == 0 and lay[-1].bot == 0
    for s in lay:
        assert s.row0 >= 0 and s.row0 + s.rows <= ny
        assert s.hi - s.lo == s.b - s.a
    with pytest.raises(ValueError):
        S.strip_layout(ny, ny + 1, 1)


def test_strip_layout_rejects_strips_thinner_than_the_halo():
    with pytest.raises(ValueError):
        S.strip_layout(10, 4, 3)


def test_combine_partials_follows_the_reduction_rule():
    nx, ny = 10, 20
    a = np.zeros(3, dtype=PARTIAL_DTYPE)
    b = np.zeros(3, dtype=PARTIAL_DTYPE)
    a[0] = (500.0, 57, 5, 6); b[0] = (500.0, 31, 3, 3)           # tie: smaller index
    a[1] = (np.nan, 1, ny, -1); b[1] = (400.0, 150, ny, -1)       # NaN never wins
    a[2] = (-1.0, nx * ny, ny, -1); b[2] = (-1.0, nx * ny, ny, -1)  # both neutral
    out = S.combine_partials([a, b], nx, ny)
    assert tuple(out[0]) == (500.0, 31, 3, 6)
    assert tuple(out[1]) == (400.0, 150, ny, -1)
    assert tuple(out[2]) == (-1.0, nx * ny, ny, -1)


# ---- halo exchange with the oracle as the strip stepper (CPU) -----------------

@pytest.mark.parametrize("parts,depth,bc", [(3, 3, 0), (2, 4, 1), (4, 1, 0)])
def test_local_strips_match_the_whole_field(parts, depth, bc):
    from oracle import oracle as O
    mat, k, T0, las, plan = _case()
    T_ref, ring_ref = O.run(T0.ravel(), k, las, bc=bc, T_D=300.0, Tm=mat.Tm)
    f = S.ShardedField.local(k, parts, depth=depth, device="cpu", T0=T0,
                             stepper=OracleStripStepper(bc=bc, Tm=mat.Tm))
    rings = f.advance(plan)
    _check(f.field().numpy().ravel(), f.partials(rings), T_ref, ring_ref)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out, depth=3, bc=0):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mat, k, T0, las, plan = _case()
        f = S.ShardedField.distributed(k, rank, world, depth=depth, device="cpu", T0=T0,
                                       stepper=OracleStripStepper(bc=bc, Tm=mat.Tm))
        rings = f.advance(plan)
        # every rank takes the same collective steps in the same order
        T = f.field().numpy()
        parts = f.partials(rings)
        out[rank] = (T, parts.tobytes(), f.strips[0])
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_exchange_halos():
    import torch.multiprocessing as mp
    from oracle import oracle as O
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(world, _free_port(), out), nprocs=world,
                       start_method="spawn", join=True)
    mat, k, T0, las, plan = _case()
    T_ref, ring_ref = O.run(T0.ravel(), k, las, Tm=mat.Tm)
    strips = [out[r][2] for r in range(world)]
    assert strips[0].b == strips[1].a and strips[0].bot == strips[1].top == 3
    for r in range(world):
        T, pb, _ = out[r]
        _check(T.ravel(), np.frombuffer(pb, dtype=PARTIAL_DTYPE), T_ref, ring_ref)
    assert out[0][1] == out[1][1]                    # every rank holds the same result


# ---- the CUDA strip kernel (GPU) ----------------------------------------------

@pytest.mark.gpu
@pytest.mark.parametrize("nx,ny,parts,depth,bc", [
    (300, 260, 3, 3, 0), (300, 260, 1, 2, 0), (129, 77, 2, 4, 1), (1024, 1030, 4, 3, 0),
    (248, 96, 5, 1, 0)])
def test_gpu_strips_equal_the_single_field(gpu, nx, ny, parts, depth, bc):
    from hedgehog_lpbf_b200.solver import Solver, ring_to_numpy
    mat, dom, k = _const(nx, ny)
    rng = np.random.default_rng(nx + ny)
    T0 = 300.0 + rng.uniform(0.0, 1500.0, size=(ny, nx))
    n = 13
    plan = PL.raster_for_steps(dom, k.dt, n, V=1.0, hatch=100e-6, n_tracks=2, angle=1.2)
    ref = Solver(k, bc=bc, T_edge=300.0, Tm=mat.Tm, depth=depth, device=gpu, T0=T0)
    ring_ref = ref.new_ring(n)
    T_ref = ref.advance(plan, ring_ref).cpu().numpy()
    f = S.ShardedField.local(k, parts, depth=depth, device=gpu, T0=T0, bc=bc, T_edge=300.0,
                             Tm=mat.Tm)
    rings = f.advance(plan)
    T = f.field().cpu().numpy()
    assert np.array_equal(T.view(np.uint64), T_ref.view(np.uint64))
    assert f.partials(rings).tobytes() == ring_to_numpy(ring_ref).tobytes()
    assert f.read_error() == 0
    # and the oracle agrees with both
    from oracle import oracle as O
    T_o, _ = O.run(T0.ravel(), k, PL.laser_array(plan), bc=bc, T_D=300.0, Tm=mat.Tm)
    assert np.max(np.abs(T.ravel() - T_o) / np.maximum(np.abs(T_o), 1.0)) <= RTOL


@pytest.mark.gpu
def test_gpu_advance_rows_rejects_bad_windows(gpu):
    import ctypes
    from hedgehog_lpbf_b200 import _lib
    L = _lib.lib()
    mat, dom, k = _const(64, 40)
    ks = S.strip_const(k, S.Strip(10, 30, 3, 3))          # 26 buffer rows
    a = torch.zeros((26, 64), dtype=torch.float64, device=gpu)
    b = torch.zeros_like(a)
    plan = PL.raster_for_steps(dom, k.dt, 4, V=1.0, hatch=100e-6, n_tracks=1)
    opts = _lib.Opts(phys=0, bc=0, T_edge=300.0, Tm=mat.Tm, depth=0, rows=0)
    s = torch.cuda.current_stream().cuda_stream

    def call(row0, lo, hi, n, phys=0):
        o = _lib.Opts(phys=phys, bc=0, T_edge=300.0, Tm=mat.Tm, depth=0, rows=0)
        rw = _lib.Rows(row0=row0, global_ny=40, lo=lo, hi=hi)
        return L.lpbf_b200_advance_rows(a.data_ptr(), b.data_ptr(), ctypes.byref(ks),
                                        plan.ctypes.data, n, ctypes.byref(o), ctypes.byref(rw),
                                        None, None, 0, s)

    assert call(7, 3, 23, 3) == 0                         # 3 halo rows each side, 3 steps
    torch.cuda.synchronize()
    assert call(7, 3, 23, 4) == -1                        # halo thinner than the steps
    assert call(7, 2, 23, 3) == -1
    assert call(7, 3, 24, 3) == -1
    assert call(0, 0, 23, 3) == 0                         # top edge of the field: no halo
    assert call(7, 3, 23, 5) == -1                        # more than 4 steps in one launch
    assert call(15, 3, 23, 3) == -1                       # strip beyond the field
    assert call(7, 3, 23, 3, phys=1) == -2                # baseline physics only
    del opts


def test_three_gloo_ranks_interior_strip():
    """An interior strip trades rows with both neighbours; fixed edges, 2 steps
    per launch."""
    import torch.multiprocessing as mp
    from oracle import oracle as O
    world = 3
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(world, _free_port(), out, 2, 1), nprocs=world,
                       start_method="spawn", join=True)
    mat, k, T0, las, plan = _case()
    T_ref, ring_ref = O.run(T0.ravel(), k, las, bc=1, T_D=300.0, Tm=mat.Tm)
    mid = out[1][2]
    assert mid.top == mid.bot == 2
    for r in range(world):
        T, pb, _ = out[r]
        _check(T.ravel(), np.frombuffer(pb, dtype=PARTIAL_DTYPE), T_ref, ring_ref)


@pytest.mark.parametrize("seed", range(6))
def test_strip_partials_combine_to_the_field_reduction(seed):
    """Random fields with planted ties and molten rows, cut into random strip
    counts: per-strip Partials (owned rows, field numbering) combined by the
    reduction rule equal the oracle's whole-field reduction."""
    from oracle import oracle as O
    rng = np.random.default_rng(seed)
    nx, ny = int(rng.integers(4, 40)), int(rng.integers(6, 60))
    Tm = 1500.0
    T = rng.choice([300.0, 900.0, 1600.0, 2000.0], size=(ny, nx), p=[0.6, 0.25, 0.1, 0.05])
    if seed % 2:
        T[:] = 300.0                                    # all tied, none molten
    parts = int(rng.integers(1, min(6, ny) + 1))
    rings = []
    for s in S.strip_layout(ny, parts, 1):
        own = T[s.a:s.b]
        tm, ag, mn, mx = O.reduce(own.ravel(), nx, s.b - s.a, Tm)
        r = np.zeros(1, dtype=PARTIAL_DTYPE)
        neutral = ag >= nx * (s.b - s.a)
        r[0] = (tm, nx * ny if neutral else ag + s.a * nx,
                ny if mx < 0 else mn + s.a, -1 if mx < 0 else mx + s.a)
        rings.append(r)
    got = S.combine_partials(rings, nx, ny)[0]
    assert tuple(got) == O.reduce(T.ravel(), nx, ny, Tm)
