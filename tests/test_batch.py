# SPDX-License-Identifier: 0BSD
"""Batched process map (lpbf_b200_batch_*): every scenario's final field and
per-step Partials are bit-identical to its own single-field run
(lpbf_b200_advance, itself held to the oracle by test_gpu_parity), whatever
the batch composition, depth, rows per task, CTAs per SM or graph replay."""
import math

import numpy as np
import pytest

from hedgehog_lpbf_b200 import params as P
from hedgehog_lpbf_b200 import plan as PL
from hedgehog_lpbf_b200 import process_map as PM

pytestmark = pytest.mark.gpu


def _const(nx, ny, Pw=200.0, V=1.0, r0=50e-6):
    mat, pr = P.benchmark_material_process(P=Pw, V=V, r0=r0)
    dom = P.Domain(Lx=(nx - 1) * 5e-6, Ly=(ny - 1) * 5e-6, nx=nx, ny=ny)
    dt = P.dt_fraction(mat, dom)
    return mat, dom, P.make_const(mat, pr, dom, dt)


def _mixed(n_steps, shapes, seed=0, random_T0=True):
    from hedgehog_lpbf_b200.batch import Scenario
    rng = np.random.default_rng(seed)
    out = []
    for nx, ny, bc in shapes:
        mat, dom, k = _const(nx, ny, Pw=100 + 300 * rng.random(), V=0.5 + 1.5 * rng.random(),
                             r0=35e-6 + 35e-6 * rng.random())
        plan = PL.raster_for_steps(dom, k.dt, n_steps, V=1.5, hatch=100e-6,
                                   n_tracks=2, angle=math.pi * rng.random())
        T0 = (300.0 + rng.uniform(0.0, 1800.0, size=(ny, nx))) if random_T0 else None
        out.append(Scenario(k=k, plan=plan, bc=bc, T_edge=300.0, Tm=mat.Tm, T0=T0))
    return out


def _single(sc, n_steps, depth=0):
    from hedgehog_lpbf_b200.solver import Solver, ring_to_numpy
    s = Solver(sc.k, bc=sc.bc, T_edge=sc.T_edge, Tm=sc.Tm, depth=depth, device="cuda:0",
               T0=sc.T0 if sc.T0 is not None else sc.k.Tamb)
    ring = s.new_ring(n_steps)
    s.advance(sc.plan[:n_steps], ring)
    return s.field.cpu().numpy(), ring_to_numpy(ring)


def _assert_same(b, scs, n_steps, refs):
    for i in range(len(scs)):
        T, ring = refs[i]
        Tb = b.field(i).cpu().numpy()
        assert np.array_equal(Tb.view(np.uint64), T.view(np.uint64)), f"scenario {i} field"
        assert b.ring(i)[:n_steps].tobytes() == ring.tobytes(), f"scenario {i} ring"


SHAPES = [(256, 256, 0), (302, 260, 0), (512, 512, 1), (130, 98, 0), (1024, 64, 1),
          (64, 700, 0), (384, 200, 1)]


@pytest.fixture(scope="module")
def mixed13(gpu):
    n = 13
    scs = _mixed(n, SHAPES, seed=3)
    refs = [_single(sc, n) for sc in scs]
    return scs, refs, n


@pytest.mark.parametrize("depth,rows,ctas,staging", [
    (3, (0, 0, 0, 0), 0, 0), (4, (12, 30, 48, 9), 2, 1), (1, (24, 24, 24, 24), 1, 2),
    (2, (96, 7, 17, 64), 0, 2), (3, (16, 40, 24, 8), 0, 2)])
def test_batch_matches_single_runs(mixed13, depth, rows, ctas, staging):
    from hedgehog_lpbf_b200.batch import Batch, batch_opts
    scs, refs, n = mixed13
    b = Batch(scs, n, opts=batch_opts(depth=depth, ctas_per_sm=ctas, rows=rows, staging=staging),
              device="cuda:0")
    b.run(0, n)
    assert b.read_error() == 0
    assert b.cur == ((n + depth - 1) // depth) % 2
    _assert_same(b, scs, n, refs)
    b.close()


def test_batch_graph_replay_and_split_runs(mixed13):
    import torch
    from hedgehog_lpbf_b200.batch import Batch, batch_opts
    scs, refs, n = mixed13
    b = Batch(scs, n, opts=batch_opts(depth=3), device="cuda:0")
    b.run(0, n, use_graph=True)
    torch.cuda.synchronize()
    _assert_same(b, scs, n, refs)
    # the same steps again from the start fields, now written into the other
    # buffer: a second graph (other parity) is captured, then one is replayed
    for _ in range(2):
        for i, sc in enumerate(scs):
            b.set_field(i, sc.T0)
        b.run(0, n, use_graph=True)
        torch.cuda.synchronize()
        _assert_same(b, scs, n, refs)
    # split into two runs with a remainder launch in the middle
    for i, sc in enumerate(scs):
        b.set_field(i, sc.T0)
    b.run(0, 7)
    b.run(7, n - 7, use_graph=True)
    _assert_same(b, scs, n, refs)
    assert b.read_error() == 0
    b.close()


def test_batch_direct_load_path(gpu):
    """An odd row length (no bulk staging) switches the batch to direct loads."""
    from hedgehog_lpbf_b200.batch import Batch, batch_opts
    n = 8
    scs = _mixed(n, [(257, 131, 0), (200, 300, 1), (96, 96, 0)], seed=5)
    refs = [_single(sc, n) for sc in scs]
    b = Batch(scs, n, opts=batch_opts(depth=3), device="cuda:0")
    b.run(0, n)
    _assert_same(b, scs, n, refs)
    b.close()


def test_batch_process_map_draws(gpu):
    """Seeded process-map draws at their full grid sides (256..2048),
    serpentine rasters at random angles, uniform 300 K start."""
    from hedgehog_lpbf_b200.batch import Batch, batch_opts
    n = 30
    scs = PM.process_map(12, n)
    assert {d.tag["draw"].side for d in scs} >= {256, 2048}
    refs = [_single(sc, n) for sc in scs]
    b = Batch(scs, n, opts=batch_opts(depth=3, rows=(12, 24, 24, 48)), device="cuda:0")
    b.run(0, n, use_graph=True)
    _assert_same(b, scs, n, refs)
    for i in range(len(scs)):
        r = b.ring(i)
        assert np.all(r["tmax"] > 300.0) and np.all(r["arg"] >= 0)
    b.close()


def test_batch_matches_oracle_small(gpu):
    from oracle import oracle as O
    from hedgehog_lpbf_b200.batch import Batch, batch_opts
    n = 9
    # mirror edges mid-strip (248 = 2 strips + 8 columns), a substrate
    # temperature other than the ambient one, fixed edges
    scs = _mixed(n, [(120, 90, 0), (200, 64, 1), (248, 96, 0), (244, 80, 0)], seed=8)
    scs[3].k.Tsub = 420.0
    refs = [O.run(np.asarray(sc.T0).ravel(), sc.k, PL.laser_array(sc.plan[:n]),
                  bc=sc.bc, T_D=sc.T_edge, Tm=sc.Tm) for sc in scs]
    for staging in (1, 2):
        b = Batch(scs, n, opts=batch_opts(depth=4, staging=staging), device="cuda:0")
        b.run(0, n)
        for i, (T_ref, ring_ref) in enumerate(refs):
            T = b.field(i).cpu().numpy().ravel()
            err = float(np.max(np.abs(T - T_ref) / np.maximum(np.abs(T_ref), 1.0)))
            assert err <= 1e-12, (staging, i, err)
            r = b.ring(i)
            assert np.array_equal(r["arg"], ring_ref["arg"])
            assert np.max(np.abs(r["tmax"] - ring_ref["tmax"]) / ring_ref["tmax"]) <= 1e-12
        b.close()


def test_batch_rejects_bad_arguments(gpu):
    import ctypes

    from hedgehog_lpbf_b200 import _lib
    from hedgehog_lpbf_b200.batch import batch_opts
    L = _lib.lib()
    arr = (_lib.Scenario * 1)()
    assert L.lpbf_b200_batch_workspace_bytes(arr, 1, 4, ctypes.byref(batch_opts(depth=5))) == 0
    h = ctypes.c_void_p()
    assert L.lpbf_b200_batch_create(arr, 1, 4, None, None, 0, None, ctypes.byref(h)) == -1
    assert not h.value


def test_autotune_trials_cache_and_tuned_batch(gpu, tmp_path):
    import json
    import time

    from hedgehog_lpbf_b200.batch import Batch, autotune, opts_dict, tune_key
    n = 12
    scs = _mixed(n, [(256, 256, 0), (600, 520, 0), (1100, 1030, 1), (300, 2050, 0)], seed=11)
    cache = str(tmp_path / "tune.json")
    o1 = autotune(scs, n, cache=cache, trial_steps=6)
    d1 = opts_dict(o1)
    assert d1["depth"] in (2, 3, 4) and d1["staging"] in (1, 2)
    assert all(r in (12, 24, 48, 96, 192, 384) for r in d1["rows"])
    doc = json.load(open(cache))
    assert tune_key(scs) in doc["entries"] and doc["entries"][tune_key(scs)]["gcells"] > 0
    t0 = time.time()
    o2 = autotune(scs, n, cache=cache, trial_steps=6)       # from the cache
    assert opts_dict(o2) == d1 and time.time() - t0 < 1.0
    refs = [_single(sc, n) for sc in scs]
    b = Batch(scs, n, opts=o1, device="cuda:0")
    b.capture(0, n)
    b.run(0, n, use_graph=True)
    _assert_same(b, scs, n, refs)
    b.close()


def test_snapshot_resume_is_bit_identical(gpu, tmp_path):
    """(snapshot, step) is a full checkpoint: stopping after step s, writing
    T_step_s.bin and resuming from it gives the uninterrupted run's field and
    Partials bit for bit."""
    from hedgehog_lpbf_b200 import checkpoint
    from hedgehog_lpbf_b200.solver import Solver, ring_to_numpy
    mat, dom, k = _const(600, 400)
    n = 40
    plan = PL.raster_for_steps(dom, k.dt, n, V=1.5, hatch=100e-6, n_tracks=2, angle=0.3)
    a = Solver(k, Tm=mat.Tm, device="cuda:0")
    ra = a.new_ring(n)
    a.advance(plan, ra)
    b = Solver(k, Tm=mat.Tm, device="cuda:0")
    rb1 = b.new_ring(17)
    b.advance(plan[:17], rb1)
    checkpoint.save(b.field, str(tmp_path), 16)
    c = checkpoint.resume(Solver(k, Tm=mat.Tm, device="cuda:0"), str(tmp_path), 16)
    rb2 = c.new_ring(n - 17)
    c.advance(plan[17:], rb2)
    assert np.array_equal(c.field.cpu().numpy().view(np.uint64), a.field.cpu().numpy().view(np.uint64))
    assert (ring_to_numpy(rb1).tobytes() + ring_to_numpy(rb2).tobytes()) == ring_to_numpy(ra).tobytes()
