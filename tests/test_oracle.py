# SPDX-License-Identifier: 0BSD
"""The oracle pinned against the reference: its committed case-0 outputs, the
golden fields of the reference's own cpu_step, its make_const and its laser
planner.  CPU only."""
import ctypes
import json
import os

import numpy as np
import pytest

from hedgehog_lpbf_b200 import params as P
from hedgehog_lpbf_b200 import plan as PL
from oracle import oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def gold():
    return np.load(os.path.join(GOLD, "ref_small.npz"))


def fmt6(v: float) -> str:
    # the reference writes metrics.csv with the default ostream precision (6)
    return "%.6g" % v


def test_case0_golden_metrics():
    """Oracle run of the reference's case 0 reproduces reference/case0/metrics.csv
    and the peaks of meta.json at the precision they were written with."""
    g = json.load(open(os.path.join(GOLD, "case0.json")))
    mat, dom = P.Material(), P.Domain()
    pr = P.apply_case("0", P.Process())
    dt = P.dt_cfl(mat, dom)
    n = int(1.5e-3 / dt)
    assert n == g["meta"]["n_steps"]
    assert fmt6(dt) == fmt6(g["meta"]["dt_s"])
    k = P.make_const(mat, pr, dom, dt)
    plan = PL.single_track(pr, dom, dt, n, snap_every=200)
    las = PL.laser_array(plan)
    T = np.full(dom.nx * dom.ny, pr.Tamb)
    rows, peak_T, peak_W = [], pr.Tamb, 0.0
    for s in range(n):
        k.x_l, k.y_l, k.q_scale = las[s]
        T = O.step(T, k)
        m = O.measure(T, dom.nx, dom.ny, dom.dy(), mat.Tm)
        peak_T = max(peak_T, m["peak_T"])
        peak_W = max(peak_W, m["W_um"])
        if plan["dump"][s]:
            rows.append([s, s * dt * 1e6, plan["x_laser_csv"][s] * 1e6, m["peak_T"], m["W_um"]])
    want = [[r["step"], r["t_us"], r["x_laser_um"], r["peakT_K"], r["W_um"]] for r in g["metrics"]]
    assert len(rows) == len(want) == 9
    for got, exp in zip(rows, want):
        assert [fmt6(v) for v in got] == [fmt6(v) for v in exp]
    assert fmt6(peak_T) == fmt6(g["meta"]["peak_T_K"])
    assert fmt6(peak_W) == fmt6(g["meta"]["peak_W_um"])


@pytest.mark.parametrize("name", ["mirror_64x48", "mirror_odd_33x17", "mirror_130x70_edge",
                                  "ext_48x40", "ext_kmult_40x24"])
def test_oracle_bit_identical_to_reference_cpu_step(gold, name):
    """The C restatement equals the reference's own cpu_step bit for bit."""
    k = O.OracleStepConst.from_buffer_copy(gold[f"{name}/const"].tobytes())
    las = gold[f"{name}/laser"]
    T, _ = O.run(gold[f"{name}/T0"], k, las, phys=int(gold[f"{name}/phys"]), with_ring=False)
    assert np.array_equal(T.view(np.uint64), gold[f"{name}/T"].view(np.uint64))


@pytest.mark.parametrize("name", ["mirror_64x48", "mirror_130x70_edge", "ext_48x40"])
def test_oracle_measure_matches_reference(gold, name):
    k = O.OracleStepConst.from_buffer_copy(gold[f"{name}/const"].tobytes())
    m = O.measure(gold[f"{name}/T"], k.nx, k.ny, k.dy, 1609.0)
    ref = gold[f"{name}/measure"]
    assert m["peak_T"] == ref[0] and m["W_um"] == ref[1] and m["W_sub_um"] == ref[2]
    assert m["x_hot"] == int(ref[3])


def test_make_const_matches_reference(gold):
    for cid in P.CASES:
        mat, dom = P.Material(), P.Domain()
        pr = P.apply_case(cid, P.Process())
        dt = P.dt_cfl(mat, dom)
        assert dt == float(gold[f"dt_case{cid}"])
        assert bytes(P.make_const(mat, pr, dom, dt)) == gold[f"const_case{cid}"].tobytes()
    mat, pr = P.benchmark_material_process()
    for n in (512, 8192):
        dom = P.square_domain(n)
        k = P.make_const(mat, pr, dom, P.dt_fraction(mat, dom))
        assert bytes(k) == gold[f"const_bench{n}"].tobytes()


def test_single_track_plan_matches_reference_build_plan(gold):
    mat, dom = P.Material(), P.Domain()
    pr = P.apply_case("0", P.Process())
    dt = P.dt_cfl(mat, dom)
    n = int(1.5e-3 / dt)
    plan = PL.single_track(pr, dom, dt, n, snap_every=200)
    ref = gold["plan_case0"].view(PL.TICK_DTYPE)
    for f in PL.TICK_DTYPE.names:
        assert np.array_equal(plan[f], ref[f]), f


def test_reduce_semantics_ties_and_nan():
    """GPU-reduce semantics: ties -> smallest flat index; NaN and values <= -1
    never win; molten rows strictly above Tm."""
    nx, ny = 7, 5
    T = np.full(nx * ny, 300.0)
    T[9] = T[30] = 2000.0          # tie: index 9 wins
    T[12] = np.nan
    tmax, arg, ymin, ymax = O.reduce(T, nx, ny, 1609.0)
    assert (tmax, arg, ymin, ymax) == (2000.0, 9, 1, 4)
    T2 = np.full(nx * ny, -5.0)
    assert O.reduce(T2, nx, ny, 0.0) == (-1.0, nx * ny, ny, -1)


def test_dirichlet_oracle_fixes_edges_and_matches_mirror_inside():
    mat, pr = P.benchmark_material_process()
    dom = P.square_domain(40)
    k = P.make_const(mat, pr, dom, P.dt_fraction(mat, dom))
    k.x_l, k.y_l, k.q_scale = 0.5 * dom.Lx, 0.5 * dom.Ly, 1.0
    T0 = np.full(40 * 40, 300.0)
    Td = O.step(T0, k, bc=1, T_D=300.0).reshape(40, 40)
    Tm = O.step(T0, k, bc=0).reshape(40, 40)
    assert np.all(Td[0] == 300.0) and np.all(Td[-1] == 300.0)
    assert np.all(Td[:, 0] == 300.0) and np.all(Td[:, -1] == 300.0)
    # one step from a uniform field: interior cells see identical neighbours
    assert np.array_equal(Td[1:-1, 1:-1], Tm[1:-1, 1:-1])


def test_reference_cpu_step_available_matches_oracle_when_built():
    """With oracle/_ref built (reference tree present), the live reference
    agrees with the oracle on a fresh random case too."""
    if not O.have_reference():
        pytest.skip("oracle/_ref not built here")
    mat, pr = P.benchmark_material_process()
    dom = P.Domain(Lx=57 * 5e-6, Ly=30 * 5e-6, nx=58, ny=31)
    k = P.make_const(mat, pr, dom, P.dt_fraction(mat, dom))
    rng = np.random.default_rng(11)
    T0 = 300.0 + rng.uniform(0, 3000, size=58 * 31)
    las = np.array([[rng.uniform(0, dom.Lx), rng.uniform(0, dom.Ly), 1.0] for _ in range(15)])
    T_o, _ = O.run(T0, k, las, with_ring=False)
    T_r = O.ref_run_plan(T0, k, las)
    assert np.array_equal(T_o, T_r)


def test_reference_steptiletask_matches_oracle_when_built():
    """The reference's StepTileTask over 64-row strips on 4 threads (hh-compat)
    equals the full-grid oracle bit for bit."""
    if not O.have_reference():
        pytest.skip("oracle/_ref not built here")
    mat, pr = P.benchmark_material_process()
    dom = P.square_domain(96)
    k = P.make_const(mat, pr, dom, P.dt_fraction(mat, dom))
    plan = PL.raster_for_steps(dom, k.dt, 12, V=1.0, hatch=100e-6, n_tracks=2)
    las = PL.laser_array(plan)
    T0 = np.full(96 * 96, 300.0)
    T_hh, wall, trace = O.ref_hh_run(T0, mat, pr, dom, k.dt, las, n_threads=4, n_tiles=3,
                                     Tm=mat.Tm, want_trace=True)
    T_o, ring = O.run(T0, k, las, Tm=mat.Tm)
    assert np.array_equal(T_hh, T_o)
    assert np.array_equal(trace, ring["tmax"])


@pytest.mark.parametrize("seed", range(5))
def test_reference_cpu_step_matches_oracle_random_cases(seed):
    """Random grids, spot paths, start fields and substrate temperatures
    (Tsub != Tamb included): the oracle equals the live reference bit for
    bit."""
    if not O.have_reference():
        pytest.skip("oracle/_ref not built here")
    rng = np.random.default_rng(100 + seed)
    nx, ny = int(rng.integers(8, 90)), int(rng.integers(4, 60))
    mat, pr = P.benchmark_material_process(P=float(rng.uniform(100, 400)),
                                           r0=float(rng.uniform(30e-6, 70e-6)))
    pr.Tsub = float(rng.choice([pr.Tamb, 420.0, 250.0]))
    pr.radiation = bool(seed % 2 == 0)
    dom = P.Domain(Lx=(nx - 1) * 5e-6, Ly=(ny - 1) * 5e-6, nx=nx, ny=ny)
    k = P.make_const(mat, pr, dom, P.dt_fraction(mat, dom))
    T0 = 300.0 + rng.uniform(0, 2500, size=nx * ny)
    n = int(rng.integers(3, 12))
    las = np.stack([rng.uniform(-0.1, 1.1, n) * dom.Lx, rng.uniform(-0.1, 1.1, n) * dom.Ly,
                    rng.choice([0.0, 0.5, 1.0], n)], axis=1)
    T_o, _ = O.run(T0, k, las, with_ring=False)
    T_r = O.ref_run_plan(T0, k, las)
    assert np.array_equal(T_o, T_r)


@pytest.mark.parametrize("case", ["uniform_raster", "warm_patch_fixed_edges", "edge_corner",
                                  "nan_and_ties"])
def test_quiet_run_bit_identical_to_full_run(case):
    """oracle.run_quiet (cells that provably stay at Tamb skipped, rows shared
    among threads) equals the full-grid oracle.run bit for bit, field and
    every per-step Partial, whatever the thread count; its probe reads the
    field after each step."""
    mat, pr = P.benchmark_material_process()
    nx, ny, n, bc = 300, 220, 240, 0
    dom = P.Domain(Lx=(nx - 1) * 5e-6, Ly=(ny - 1) * 5e-6, nx=nx, ny=ny)
    k = P.make_const(mat, pr, dom, P.dt_fraction(mat, dom))
    T0 = np.full(nx * ny, 300.0)
    plan = PL.raster_for_steps(dom, k.dt, n, V=1.0, hatch=100e-6, n_tracks=3, angle=0.3)
    if case == "warm_patch_fixed_edges":
        bc = 1
        rng = np.random.default_rng(4)
        T0.reshape(ny, nx)[40:90, 200:260] = 300.0 + rng.uniform(0.0, 900.0, (50, 60))
    elif case == "edge_corner":
        plan = PL.raster(dom, k.dt, n, V=1.0, hatch=100e-6, track_len=0.6e-3, n_tracks=3,
                         center=(0.05e-3, 0.08e-3))
    elif case == "nan_and_ties":
        T0.reshape(ny, nx)[100, 50] = np.nan
        T0.reshape(ny, nx)[[10, 30], [20, 20]] = 5000.0   # two equal peaks
        plan["q_scale"][::3] = 0.0
    las = PL.laser_array(plan)
    T_ref, ring_ref = O.run(T0, k, las, bc=bc, Tm=mat.Tm)
    probe = np.arange(n, dtype=np.int64) * 211 % (nx * ny)
    for threads in (1, 4):
        T, ring, pv = O.run_quiet(T0, k, las, bc=bc, Tm=mat.Tm, threads=threads, probe=probe)
        assert np.array_equal(T.view(np.uint64), T_ref.view(np.uint64)), threads
        assert ring.tobytes() == ring_ref.tobytes(), threads
    assert np.array_equal(pv[-1:], T_ref[probe[-1:]], equal_nan=True)
    with pytest.raises(ValueError):
        k2 = P.make_const(mat, pr, dom, k.dt)
        k2.Tsub = 420.0
        O.run_quiet(T0, k2, las[:2], Tm=mat.Tm)
