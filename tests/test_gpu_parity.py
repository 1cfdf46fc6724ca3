# SPDX-License-Identifier: 0BSD
"""GPU parity: the sm_100a kernels through the C-ABI against the oracle (the
reference's CPU step restated in C, itself pinned bit-for-bit to the
reference in test_oracle.py).

Tolerance: fields within max relative error 1e-12 (denominator max(|T|, 1),
the reference --check's definition); reductions exact on identical fields;
per-step Partials of independently advanced fields: peak T within 1e-12,
molten-row extents exact, argmax a maximizer within 1e-12.
"""
import ctypes

import numpy as np
import pytest

from hedgehog_lpbf_b200 import params as P
from hedgehog_lpbf_b200 import plan as PL
from oracle import oracle as O

pytestmark = pytest.mark.gpu
RTOL = 1e-12


def torch_mod():
    import torch
    return torch


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1.0))) if a.size else 0.0


def bench_const(nx, ny, dx=5e-6):
    mat, pr = P.benchmark_material_process()
    dom = P.Domain(Lx=(nx - 1) * dx, Ly=(ny - 1) * dx, nx=nx, ny=ny)
    return mat, pr, dom, P.make_const(mat, pr, dom, P.dt_fraction(mat, dom))


def solver(k, **kw):
    from hedgehog_lpbf_b200.solver import Solver
    return Solver(k, device="cuda:0", **kw)


def tick_plan(las):
    plan = np.zeros(len(las), dtype=PL.TICK_DTYPE)
    plan["step"] = np.arange(len(las))
    plan["x_l"], plan["y_l"], plan["q_scale"] = las[:, 0], las[:, 1], las[:, 2]
    return plan


def check_partials(ring_gpu, ring_ref, T_ref_last=None, nx=None):
    assert len(ring_gpu) == len(ring_ref)
    assert rel_err(ring_gpu["tmax"], ring_ref["tmax"]) <= RTOL
    assert np.array_equal(ring_gpu["ymin"], ring_ref["ymin"])
    assert np.array_equal(ring_gpu["ymax"], ring_ref["ymax"])
    if T_ref_last is not None:
        a = int(ring_gpu["arg"][-1])
        assert abs(T_ref_last.ravel()[a] - ring_ref["tmax"][-1]) <= RTOL * ring_ref["tmax"][-1]


LASERS = {
    "centre": lambda dom: (0.5 * dom.Lx, 0.5 * dom.Ly, 1.0),
    "corner": lambda dom: (0.0, 0.0, 1.0),
    "far_edge": lambda dom: (dom.Lx, 0.37 * dom.Ly, 1.0),
    "off": lambda dom: (0.5 * dom.Lx, 0.5 * dom.Ly, 0.0),
}


@pytest.mark.parametrize("shape", [(8, 8), (33, 17), (64, 48), (130, 70), (250, 251), (258, 200)])
@pytest.mark.parametrize("bc", [0, 1])
@pytest.mark.parametrize("laser", list(LASERS))
def test_one_step_vs_oracle(gpu, shape, bc, laser):
    nx, ny = shape
    mat, pr, dom, k = bench_const(nx, ny)
    rng = np.random.default_rng(nx * 1000 + ny)
    T0 = 300.0 + rng.uniform(0.0, 2500.0, size=nx * ny)
    las = np.array([LASERS[laser](dom)])
    T_ref, ring_ref = O.run(T0, k, las, bc=bc, T_D=300.0, Tm=mat.Tm)
    s = solver(k, bc=bc, T_edge=300.0, Tm=mat.Tm, depth=1, T0=T0)
    ring = s.new_ring(1)
    T = s.advance(tick_plan(las), ring).cpu().numpy()
    from hedgehog_lpbf_b200.solver import ring_to_numpy
    assert rel_err(T, T_ref) <= RTOL
    check_partials(ring_to_numpy(ring), ring_ref, T_ref, nx)


@pytest.mark.parametrize("shape", [(300, 260), (129, 77)])
@pytest.mark.parametrize("bc", [0, 1])
def test_depths_bit_identical_and_match_oracle(gpu, shape, bc):
    """K steps per launch (1..4) and the row-chunk size change nothing: every
    cell is evaluated by the same expression, so fields are bit-identical."""
    from hedgehog_lpbf_b200.solver import ring_to_numpy
    nx, ny = shape
    mat, pr, dom, k = bench_const(nx, ny)
    rng = np.random.default_rng(5)
    T0 = 300.0 + rng.uniform(0.0, 1500.0, size=nx * ny)
    n = 13
    las = np.stack([np.linspace(0.1, 0.9, n) * dom.Lx, np.full(n, 0.45 * dom.Ly),
                    (np.arange(n) % 4 != 3).astype(float)], axis=1)
    plan = tick_plan(las)
    T_ref, ring_ref = O.run(T0, k, las, bc=bc, T_D=300.0, Tm=mat.Tm)
    results = []
    for depth in (1, 2, 3, 4):
        for rows in (0, 16):
            s = solver(k, bc=bc, T_edge=300.0, Tm=mat.Tm, depth=depth, rows=rows, T0=T0)
            ring = s.new_ring(n)
            T = s.advance(plan, ring).cpu().numpy()
            results.append((depth, rows, T, ring_to_numpy(ring)))
            assert s.read_error() == 0
    T1, r1 = results[0][2], results[0][3]
    for depth, rows, T, r in results[1:]:
        assert np.array_equal(T.view(np.uint64), T1.view(np.uint64)), (depth, rows)
        assert r.tobytes() == r1.tobytes(), (depth, rows)
    assert rel_err(T1, T_ref) <= RTOL
    check_partials(r1, ring_ref, T_ref, nx)


@pytest.mark.parametrize("bc", [1, 0])
def test_512_full_run_2000_steps(gpu, bc):
    """512 x 512, dx = 5 um, dt = 0.2 dx^2/alpha, 2000 steps of the reference's
    single-track law (200 W, 1 m/s, r0 = 50 um); bc 1 = Dirichlet 300 K edges."""
    from hedgehog_lpbf_b200.solver import ring_to_numpy
    mat, pr, dom, k = bench_const(512, 512)
    plan = PL.single_track(pr, dom, k.dt, 2000)
    T0 = np.full(512 * 512, 300.0)
    T_ref, ring_ref = O.run(T0, k, PL.laser_array(plan), bc=bc, T_D=300.0, Tm=mat.Tm)
    s = solver(k, bc=bc, T_edge=300.0, Tm=mat.Tm, T0=T0)
    ring = s.new_ring(2000)
    T = s.advance(plan, ring).cpu().numpy()
    err = rel_err(T, T_ref)
    print(f"512^2 x 2000 bc={bc}: max rel err {err:.3e}")
    assert err <= RTOL
    check_partials(ring_to_numpy(ring), ring_ref, T_ref, 512)


def test_extended_physics_vs_oracle(gpu):
    from hedgehog_lpbf_b200.solver import ring_to_numpy
    mat, pr, dom, k = bench_const(96, 80)
    k.kmult = 2.5
    k.dt = 0.5 * k.dt
    rng = np.random.default_rng(3)
    T0 = 300.0 + rng.uniform(0.0, 2000.0, size=96 * 80)
    n = 20
    las = np.stack([np.linspace(0.2, 0.8, n) * dom.Lx, np.full(n, 0.5 * dom.Ly), np.ones(n)], 1)
    for bc in (0, 1):
        T_ref, ring_ref = O.run(T0, k, las, phys=1, bc=bc, T_D=300.0, Tm=mat.Tm)
        s = solver(k, phys=1, bc=bc, T_edge=300.0, Tm=mat.Tm, T0=T0)
        ring = s.new_ring(n)
        T = s.advance(tick_plan(las), ring).cpu().numpy()
        assert rel_err(T, T_ref) <= RTOL
        check_partials(ring_to_numpy(ring), ring_ref, T_ref, 96)


@pytest.mark.parametrize("kmult", [1.0, 2.5])
@pytest.mark.parametrize("bc", [0, 1])
def test_extended_physics_table_segments_vs_oracle(gpu, kmult, bc):
    """Extended physics on a field whose cells sit in every segment of the
    Mills tables, on the table temperatures themselves and on both ends of
    the mushy range (where k_enh and the latent heat switch), with the laser
    crossing strip and row-chunk boundaries: every step against the oracle."""
    from hedgehog_lpbf_b200.solver import ring_to_numpy
    nx, ny = 301, 203
    mat, pr, dom, k = bench_const(nx, ny)
    k.kmult = kmult
    k.dt = 0.25 * k.dt              # stable for k up to 2.5 x 29.6 W/m/K
    rng = np.random.default_rng(int(kmult * 10) + bc)
    T0 = rng.uniform(250.0, 2600.0, size=nx * ny)
    pts = np.array([298, 473, 673, 873, 1073, 1273, 1473, 1533, 1609], dtype=np.float64)
    idx = rng.choice(nx * ny, size=4 * len(pts), replace=False)
    T0[idx] = np.concatenate([pts, np.nextafter(pts, 0.0), np.nextafter(pts, 1e9), pts + 0.5])
    n = 12
    las = np.stack([np.linspace(0.05, 0.95, n) * dom.Lx, np.linspace(0.3, 0.6, n) * dom.Ly,
                    (np.arange(n) % 5 != 4).astype(float)], axis=1)
    T_ref, ring_ref = O.run(T0, k, las, phys=1, bc=bc, T_D=300.0, Tm=mat.Tm)
    s = solver(k, phys=1, bc=bc, T_edge=300.0, Tm=mat.Tm, T0=T0)
    ring = s.new_ring(n)
    T = s.advance(tick_plan(las), ring).cpu().numpy()
    assert rel_err(T, T_ref) <= RTOL
    check_partials(ring_to_numpy(ring), ring_ref, T_ref, nx)


# ---- the reference's five launch wrappers ---------------------------------

def _stream():
    return torch_mod().cuda.current_stream().cuda_stream


@pytest.mark.parametrize("phys", [0, 1])
@pytest.mark.parametrize("shape", [(240, 120), (257, 131), (1000, 64)])
def test_reference_symbols(gpu, phys, shape):
    torch = torch_mod()
    from hedgehog_lpbf_b200 import _lib
    L = _lib.lib()
    nx, ny = shape
    mat, pr, dom, k = bench_const(nx, ny)
    if phys:
        k.dt = 0.5 * k.dt
    k.x_l, k.y_l, k.q_scale = 0.3 * dom.Lx, 0.6 * dom.Ly, 1.0
    rng = np.random.default_rng(nx)
    T0 = 300.0 + rng.uniform(0.0, 2200.0, size=nx * ny)
    T0[5] = T0[nx * ny - 3] = 9000.0                      # a tie for the argmax
    Tin = torch.tensor(T0, device=gpu)
    Tout = torch.empty_like(Tin)
    Tout2 = torch.empty_like(Tin)
    T_ref = O.step(T0, k, phys=phys)
    # step
    L.lpbf_launch_step(Tin.data_ptr(), Tout.data_ptr(), ctypes.byref(k), phys, _stream())
    torch.cuda.synchronize()
    T1 = Tout.cpu().numpy()
    assert rel_err(T1, T_ref) <= RTOL
    # reduce + finalize on the same field: exact
    nb = 256
    parts = torch.zeros(nb * 24, dtype=torch.uint8, device=gpu)
    glob = torch.zeros(24, dtype=torch.uint8, device=gpu)
    L.lpbf_launch_reduce(Tout.data_ptr(), nx, ny, mat.Tm, parts.data_ptr(), nb, _stream())
    L.lpbf_launch_reduce_finalize(parts.data_ptr(), nb, nx, ny, glob.data_ptr(), _stream())
    g = glob.cpu().numpy().view(O.PARTIAL_DTYPE)[0]
    assert (g["tmax"], g["arg"], g["ymin"], g["ymax"]) == O.reduce(T1, nx, ny, mat.Tm)
    # fused step + reduce over the reference's partial count
    nparts = ((nx + 15) // 16) * ((ny + 15) // 16)
    fparts = torch.full((nparts * 24,), 0xAB, dtype=torch.uint8, device=gpu)   # garbage
    L.lpbf_launch_step_reduce(Tin.data_ptr(), Tout2.data_ptr(), ctypes.byref(k), phys, mat.Tm,
                              fparts.data_ptr(), _stream())
    L.lpbf_launch_reduce_finalize(fparts.data_ptr(), nparts, nx, ny, glob.data_ptr(), _stream())
    torch.cuda.synchronize()
    T2 = Tout2.cpu().numpy()
    assert np.array_equal(T2.view(np.uint64), T1.view(np.uint64))
    g2 = glob.cpu().numpy().view(O.PARTIAL_DTYPE)[0]
    assert (g2["tmax"], g2["arg"], g2["ymin"], g2["ymax"]) == O.reduce(T1, nx, ny, mat.Tm)
    # hot column
    col = torch.empty(ny, dtype=torch.float64, device=gpu)
    L.lpbf_launch_extract_col(Tout2.data_ptr(), nx, ny, glob.data_ptr(), col.data_ptr(), _stream())
    torch.cuda.synchronize()
    x_hot = int(g2["arg"]) % nx
    assert np.array_equal(col.cpu().numpy(), T1.reshape(ny, nx)[:, x_hot])


def test_reduce_tie_and_nan_semantics(gpu):
    torch = torch_mod()
    from hedgehog_lpbf_b200 import _lib
    L = _lib.lib()
    nx, ny = 301, 97
    T = np.full(nx * ny, 300.0)
    T[7000] = T[123] = T[29000] = 5000.0
    T[50] = np.nan
    T[51] = np.inf * 0.0 if False else 4999.0
    d = torch.tensor(T, device=gpu)
    for nb in (1, 7, 256, 4096):
        parts = torch.zeros(nb * 24, dtype=torch.uint8, device=gpu)
        glob = torch.zeros(24, dtype=torch.uint8, device=gpu)
        L.lpbf_launch_reduce(d.data_ptr(), nx, ny, 1609.0, parts.data_ptr(), nb, _stream())
        L.lpbf_launch_reduce_finalize(parts.data_ptr(), nb, nx, ny, glob.data_ptr(), _stream())
        g = glob.cpu().numpy().view(O.PARTIAL_DTYPE)[0]
        assert (g["tmax"], g["arg"], g["ymin"], g["ymax"]) == O.reduce(T, nx, ny, 1609.0)


def test_large_grid_depth_equivalence_and_oracle(gpu):
    """8192 x 8192: four steps with the laser on the grid; depth 4 equals
    depth 1 bit for bit and both match the oracle."""
    from hedgehog_lpbf_b200.solver import ring_to_numpy
    n = 8192
    mat, pr, dom, k = bench_const(n, n)
    plan = PL.raster_for_steps(dom, k.dt, 4, V=1.0, hatch=100e-6, n_tracks=1)
    T0 = np.full(n * n, 300.0)
    T0[: n * 64] = 900.0                                   # a warm band: non-trivial stencil
    T_ref, ring_ref = O.run(T0, k, PL.laser_array(plan), Tm=mat.Tm)
    out = []
    for depth in (4, 1):
        s = solver(k, Tm=mat.Tm, depth=depth, T0=T0)
        ring = s.new_ring(4)
        T = s.advance(plan, ring).cpu().numpy()
        out.append((T, ring_to_numpy(ring)))
        del s
    assert np.array_equal(out[0][0].view(np.uint64), out[1][0].view(np.uint64))
    assert out[0][1].tobytes() == out[1][1].tobytes()
    assert rel_err(out[0][0], T_ref) <= RTOL
    check_partials(out[0][1], ring_ref, T_ref, n)


def test_cuda_graph_capture_replays_advance(gpu):
    torch = torch_mod()
    from hedgehog_lpbf_b200.solver import ring_to_numpy
    mat, pr, dom, k = bench_const(512, 384)
    plan = PL.single_track(pr, dom, k.dt, 16)
    eager = solver(k, Tm=mat.Tm, depth=4)
    r_e = eager.new_ring(16)
    eager.advance(plan, r_e)
    s = solver(k, Tm=mat.Tm, depth=4)
    ring = s.new_ring(16)
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    g = torch.cuda.CUDAGraph()
    start = s.cur
    with torch.cuda.stream(side):
        with torch.cuda.graph(g, stream=side):
            s.advance(plan, ring, stream=side)
    s.cur = start
    s.set_field(300.0)
    g.replay()
    torch.cuda.synchronize()
    s.cur = 1 - start if eager.launches(16) % 2 else start
    assert np.array_equal(s.field.cpu().numpy(), eager.field.cpu().numpy())
    assert ring_to_numpy(ring).tobytes() == ring_to_numpy(r_e).tobytes()


def _const_tsub(nx, ny, Tsub):
    mat, pr = P.benchmark_material_process()
    pr.Tsub = Tsub
    dom = P.Domain(Lx=(nx - 1) * 5e-6, Ly=(ny - 1) * 5e-6, nx=nx, ny=ny)
    return mat, pr, dom, P.make_const(mat, pr, dom, P.dt_fraction(mat, dom))


@pytest.mark.parametrize("bc", [0, 1])
def test_substrate_temperature_differs_from_ambient(gpu, bc):
    """Tsub != Tamb: convection and substrate conduction pull towards different
    temperatures, so the two linear loss terms stay separate (the reference's
    q_top / q_bot)."""
    from hedgehog_lpbf_b200.solver import ring_to_numpy
    nx, ny = 300, 260
    mat, pr, dom, k = _const_tsub(nx, ny, 420.0)
    rng = np.random.default_rng(21)
    T0 = 300.0 + rng.uniform(0.0, 1500.0, size=nx * ny)
    n = 9
    plan = PL.raster_for_steps(dom, k.dt, n, V=1.0, hatch=100e-6, n_tracks=2, angle=0.4)
    T_ref, ring_ref = O.run(T0, k, PL.laser_array(plan), bc=bc, T_D=300.0, Tm=mat.Tm)
    for depth in (1, 3, 4):
        s = solver(k, bc=bc, T_edge=300.0, Tm=mat.Tm, depth=depth, T0=T0)
        ring = s.new_ring(n)
        T = s.advance(plan, ring).cpu().numpy()
        assert rel_err(T, T_ref) <= RTOL, depth
        check_partials(ring_to_numpy(ring), ring_ref, T_ref, nx)


@pytest.mark.parametrize("nx", [4, 8, 116, 120, 124, 128, 244, 248, 252, 364])
def test_mirror_edge_strips(gpu, nx):
    """Mirror edges on the fast body: for every position of the right edge
    inside a strip (the lane past the field anywhere from lane 1 to beyond
    the strip) and fields narrower than one strip, with the laser crossing
    both side edges, depths 1..4 agree bit for bit and match the oracle."""
    from hedgehog_lpbf_b200.solver import ring_to_numpy
    ny = 90
    mat, pr, dom, k = bench_const(nx, ny)
    rng = np.random.default_rng(nx)
    T0 = 300.0 + rng.uniform(0.0, 1500.0, size=nx * ny)
    n = 10
    xs = np.linspace(-0.05, 1.05, n) * dom.Lx
    las = np.stack([xs, np.linspace(0.3, 0.7, n) * dom.Ly, np.ones(n)], axis=1)
    plan = tick_plan(las)
    T_ref, ring_ref = O.run(T0, k, las, Tm=mat.Tm)
    first = None
    for depth in (1, 2, 3, 4):
        for rows in (0, 8):
            s = solver(k, Tm=mat.Tm, depth=depth, rows=rows, T0=T0)
            ring = s.new_ring(n)
            T = s.advance(plan, ring).cpu().numpy()
            r = ring_to_numpy(ring)
            if first is None:
                first = (T, r)
                assert rel_err(T, T_ref) <= RTOL
                check_partials(r, ring_ref, T_ref, nx)
            else:
                assert np.array_equal(T.view(np.uint64), first[0].view(np.uint64)), (depth, rows)
                assert r.tobytes() == first[1].tobytes(), (depth, rows)


def test_square_and_rectangular_cells(gpu):
    """Square cells (ax == ay) take the one-Laplacian form of the update,
    rectangular ones the two-term form; both match the oracle, and a batch
    holding one of each equals their single-field runs bit for bit."""
    from hedgehog_lpbf_b200.batch import Batch, Scenario, batch_opts
    from hedgehog_lpbf_b200.solver import ring_to_numpy
    mat, pr = P.benchmark_material_process()
    nx, ny, n = 256, 200, 9
    scs, singles = [], []
    for dy in (5e-6, 6.5e-6):
        dom = P.Domain(Lx=(nx - 1) * 5e-6, Ly=(ny - 1) * dy, nx=nx, ny=ny)
        k = P.make_const(mat, pr, dom, P.dt_fraction(mat, dom))   # dx = 5 um: stable for dy >= dx
        assert (k.inv_dx2 == k.inv_dy2) == (dy == 5e-6)
        rng = np.random.default_rng(int(dy * 1e7))
        T0 = 300.0 + rng.uniform(0.0, 1500.0, size=(ny, nx))
        plan = PL.raster_for_steps(dom, k.dt, n, V=1.0, hatch=100e-6, n_tracks=2, angle=0.7)
        T_ref, ring_ref = O.run(T0.ravel(), k, PL.laser_array(plan), Tm=mat.Tm)
        s = solver(k, Tm=mat.Tm, depth=3, T0=T0)
        ring = s.new_ring(n)
        T = s.advance(plan, ring).cpu().numpy()
        assert rel_err(T, T_ref) <= RTOL
        check_partials(ring_to_numpy(ring), ring_ref, T_ref, nx)
        scs.append(Scenario(k=k, plan=plan, Tm=mat.Tm, T0=T0))
        singles.append((T, ring_to_numpy(ring)))
    b = Batch(scs, n, opts=batch_opts(depth=3), device="cuda:0")
    b.run(0, n)
    for i, (T, ring) in enumerate(singles):
        assert np.array_equal(b.field(i).cpu().numpy().view(np.uint64), T.view(np.uint64))
        assert b.ring(i)[:n].tobytes() == ring.tobytes()
    b.close()


def test_run_many_streams_independent_runs(gpu):
    """Solver.run_many: each run equals its own advance from its own host
    field, whatever the overlap of the copies."""
    torch = torch_mod()
    from hedgehog_lpbf_b200.solver import ring_to_numpy
    mat, pr, dom, k = bench_const(300, 260)
    rng = np.random.default_rng(11)
    n_runs, n = 4, 7
    ins = [torch.tensor(300.0 + rng.uniform(0.0, 1500.0, size=(260, 300))).pin_memory()
           for _ in range(n_runs)]
    plans = [PL.raster_for_steps(dom, k.dt, n, V=1.0, hatch=100e-6, n_tracks=2, angle=0.3 * i)
             for i in range(n_runs)]
    outs = [torch.empty((260, 300), dtype=torch.float64).pin_memory() for _ in range(n_runs)]
    rings = [torch.empty(24 * n, dtype=torch.uint8).pin_memory() for _ in range(n_runs)]
    s = solver(k, Tm=mat.Tm, depth=3)
    s.run_many(ins, plans, outs, rings)
    for i in range(n_runs):
        ref = solver(k, Tm=mat.Tm, depth=3, T0=ins[i].numpy())
        r = ref.new_ring(n)
        T = ref.advance(plans[i], r).cpu().numpy()
        assert np.array_equal(outs[i].numpy().view(np.uint64), T.view(np.uint64)), i
        assert rings[i].numpy().tobytes() == ring_to_numpy(r).tobytes(), i
