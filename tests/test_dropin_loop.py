# SPDX-License-Identifier: 0BSD
"""The reference's per-step call sequence over this library's drop-in C-ABI
(hedgehog_lpbf_b200.dropin: lpbf_launch_step / _reduce / _reduce_finalize /
_step_reduce / _extract_col, as the reference's GpuStepTask batch loop calls
them) against the multi-step entry point: the same field and the same
per-step Partials, bit for bit, through a raster that melts, on a small
field and on the bench's 8192^2 one."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("side,steps", [(520, 300), (8192, 448)])
@pytest.mark.parametrize("fused", [False, True])
def test_reference_call_sequence_matches_multistep(gpu, fused, side, steps):
    import torch
    from hedgehog_lpbf_b200 import dropin
    from hedgehog_lpbf_b200 import params as P
    from hedgehog_lpbf_b200 import plan as PL
    from hedgehog_lpbf_b200.solver import Solver, ring_to_numpy
    mat, pr = P.benchmark_material_process()
    dom = P.square_domain(side)
    k = P.make_const(mat, pr, dom, P.dt_fraction(mat, dom))
    plan = PL.raster_for_steps(dom, k.dt, steps, V=1.0, hatch=100e-6, n_tracks=10)
    r = dropin.run(k, dom, plan, mat.Tm, fused=fused, batch=64, device="cuda:0")
    s = Solver(k, Tm=mat.Tm, device="cuda:0", T0=300.0)
    ring = s.new_ring(len(plan))
    s.advance(plan, ring)
    torch.cuda.synchronize()
    ref = ring_to_numpy(ring)
    assert np.max(ref["tmax"]) > mat.Tm            # the raster melts
    assert torch.equal(r["field"], s.field)
    assert r["partials"].tobytes() == ref.tobytes()
