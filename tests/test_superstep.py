# SPDX-License-Identifier: 0BSD
"""The learned super-stepper in use: training on solver trajectories lowers
the held-out error below both the untrained network and predicting no
change (what the trained network gains over the method without it), and
the in-loop FP64 judge rolls the laser window back to the FP64 solution
whenever the network misses the tolerance."""
import math

import numpy as np
import pytest

from hedgehog_lpbf_b200 import params as P
from hedgehog_lpbf_b200 import plan as PL

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small_training(gpu):
    from hedgehog_lpbf_b200.superstep import evaluate, make_dataset, train
    from hedgehog_lpbf_b200.surrogate import Net, init_params
    ds = make_dataset(4, 128, side=512, first_index=0)
    held = make_dataset(1, 128, side=512, first_index=100000)
    untrained = Net(init_params(0), device="cuda:0")
    before = evaluate(untrained, held, patch=128, n=32)
    net = Net(init_params(0), device="cuda:0")
    hist = train(net, ds, 300, batch=16, patch=128, seed=0, log_every=100)
    after = evaluate(net, held, patch=128, n=32)
    return net, untrained, before, after, hist


def test_training_beats_untrained_and_no_change(small_training):
    _, _, before, after, hist = small_training
    assert hist[-1]["loss"] < hist[0]["loss"]
    assert after["rms_K"] < 0.5 * after["no_change_rms_K"], after
    assert after["rms_K"] < 0.5 * before["rms_K"], (before, after)
    print(f"held-out rms: untrained {before['rms_K']:.2f} K, no change "
          f"{after['no_change_rms_K']:.2f} K, trained {after['rms_K']:.2f} K")


def _case(n=512, steps=256):
    mat, pr = P.benchmark_material_process()
    dom = P.square_domain(n)
    k = P.make_const(mat, pr, dom, P.dt_fraction(mat, dom))
    plan = PL.raster_for_steps(dom, k.dt, steps, V=1.0, hatch=100e-6, n_tracks=2, angle=0.4)
    return mat, k, plan


def test_judge_rolls_back_to_fp64_in_the_window(small_training):
    import torch
    from hedgehog_lpbf_b200.solver import Solver
    from hedgehog_lpbf_b200.superstep import run_hybrid
    net, untrained, *_ = small_training
    mat, k, plan = _case()
    T0 = np.full(k.nx * k.ny, 300.0)
    s = Solver(k, Tm=mat.Tm, device="cuda:0")
    s.advance(plan)
    T_ref = s.field.cpu().numpy()
    # a tolerance of 0 K rolls back every window: the hybrid then equals the
    # FP64 judge's window solution there
    # (guard off: the whole-field FP64 redo would hide the networks' own
    # errors outside the windows, which this compares)
    T_u, rec_u = run_hybrid(untrained, k, plan, T0, 256, judge_every=4, tol_K=0.0, guard=False)
    assert rec_u["rolled_back"] == rec_u["judged"] == 4
    T_t, rec_t = run_hybrid(net, k, plan, T0, 256, judge_every=4, tol_K=5.0, guard=False)
    assert rec_t["judged"] == 4
    # the trained network's hybrid field is closer to plain FP64 outside the
    # last window than the untrained one's (no rollback hides it there)
    err_t = float(np.abs(T_t.cpu().numpy() - T_ref).max())
    err_u = float(np.abs(T_u.cpu().numpy() - T_ref).max())
    print(f"hybrid max |dT| vs FP64: trained {err_t:.1f} K (rollbacks {rec_t['rolled_back']}), "
          f"untrained {err_u:.1f} K")
    assert err_t < err_u
    assert torch.isfinite(T_t).all()
    # with the guard on, the field stays within the maximum-principle range
    # (its lower end may move down by tol_K per block)
    T_g, rec_g = run_hybrid(net, k, plan, T0, 256, judge_every=4, tol_K=5.0)
    assert rec_g["judged"] == 4
    assert torch.isfinite(T_g).all()
    assert float(T_g.min()) >= 300.0 - 5.0 * rec_g["judged"], rec_g


def test_non_finite_block_is_redone_in_fp64(gpu):
    """A network whose every parameter is NaN makes the whole field NaN after
    each block of super-steps; the loop then redoes each block from its start
    with the FP64 solver over the whole field, so the run ends on the plain
    FP64 field."""
    import torch
    from hedgehog_lpbf_b200.solver import Solver
    from hedgehog_lpbf_b200.superstep import run_hybrid
    from hedgehog_lpbf_b200.surrogate import Net, init_params
    mat, k, plan = _case()
    net = Net(init_params(0), device="cuda:0")
    net.set_params(np.full(net.np, np.nan, dtype=np.float32))
    T0 = np.full(k.nx * k.ny, 300.0)
    s = Solver(k, Tm=mat.Tm, device="cuda:0")
    s.advance(plan)
    T, rec = run_hybrid(net, k, plan, T0, 256, judge_every=4, tol_K=5.0, Tm=mat.Tm)
    assert rec["full_fp64_blocks"] == rec["judged"] == 4
    assert torch.isfinite(T).all()
    # the judge's box solution may replace a window; it differs from the
    # whole-field solution only through the box edges, far below this bound
    err = float((T - s.field).abs().max())
    assert err < 1e-3, err
