# SPDX-License-Identifier: 0BSD
"""The FP64 restatement of the super-stepper network (oracle/surrogate_ref)
checked against central finite differences: it is the gradient checker of
the tensor-core kernels, so it is pinned first (no GPU)."""
import numpy as np

from oracle import surrogate_ref as R


def test_reference_gradients_match_finite_differences():
    ps = R.init_params(0)
    rng = np.random.default_rng(0)
    ps = [(w, rng.normal(0, 0.05, b.shape)) for w, b in ps]
    x = rng.normal(size=(1, 5, 7, 4))
    t = rng.normal(size=(1, 5, 7))
    _, g = R.loss_and_grads(ps, x, t)
    e = 1e-6
    for li, idx in [(0, (3, 4, 1)), (1, (7, 8, 30)), (2, (0, 0, 0)), (3, (31, 5, 9)),
                    (4, (0, 2, 17))]:
        w = ps[li][0]
        w[idx] += e
        lp, _ = R.loss_and_grads(ps, x, t)
        w[idx] -= 2 * e
        lm, _ = R.loss_and_grads(ps, x, t)
        w[idx] += e
        fd = (lp - lm) / (2 * e)
        assert abs(fd - g[li][0][idx]) <= 1e-6 * max(1e-3, abs(fd)), (li, fd, g[li][0][idx])
    for li in range(5):
        b = ps[li][1]
        b[0] += e
        lp, _ = R.loss_and_grads(ps, x, t)
        b[0] -= 2 * e
        lm, _ = R.loss_and_grads(ps, x, t)
        b[0] += e
        assert abs((lp - lm) / (2 * e) - g[li][1][0]) <= 1e-6 * max(1e-3, abs(g[li][1][0]))


def test_flip_transpose_is_the_adjoint():
    rng = np.random.default_rng(1)
    w = rng.normal(size=(32, 9, 4))
    x = rng.normal(size=(2, 4, 6, 4))
    g = rng.normal(size=(2, 4, 6, 32))
    assert abs(np.sum(R.conv3x3(x, w) * g) - np.sum(x * R.conv3x3_input_grad(g, w))) < 1e-6


def test_adamw_first_step_is_sign_like():
    p = np.array([1.0, -2.0, 3.0])
    g = np.array([0.5, -1e-3, 0.0])
    p1, m, v = R.adamw(p, g, np.zeros(3), np.zeros(3), 1, lr=1e-2, wd=0.0)
    assert np.allclose(p1[:2], p[:2] - 1e-2 * np.sign(g[:2]), atol=1e-7)
    assert p1[2] == p[2]


def test_judge_gates_with_host_side_fault_injection():
    """The rollback gates of the in-loop judge on CPU tensors: a window that
    matches passes; 6 K off at one cell, a 3 % melt-area change, or a NaN
    roll back; 4 K off with the same melt area does not."""
    import torch
    from hedgehog_lpbf_b200.superstep import judge
    rng = np.random.default_rng(0)
    ref = torch.tensor(300.0 + 1700.0 * rng.random((64, 80)))
    Tm = 1700.0
    assert judge(ref.clone(), ref, 5.0, 0.02, Tm)[2] is False
    got = ref.clone()
    cool = int(torch.nonzero(ref < Tm - 50)[0][0]), int(torch.nonzero(ref < Tm - 50)[0][1])
    got[cool] += 4.0
    d, a, back = judge(got, ref, 5.0, 0.02, Tm)
    assert abs(d - 4.0) < 1e-9 and a == 0.0 and back is False
    got[cool] += 2.0
    assert judge(got, ref, 5.0, 0.02, Tm)[2] is True
    # melt area: push 3 % of the molten cells below Tm by a little (< 5 K)
    got = ref.clone()
    hot = torch.nonzero((ref > Tm) & (ref < Tm + 2.0))
    molten = int((ref > Tm).sum())
    need = int(np.ceil(0.03 * molten))
    if len(hot) < need:                      # make enough cells sit just above Tm
        flat = torch.nonzero(ref > Tm)[:need]
        ref[flat[:, 0], flat[:, 1]] = Tm + 1.0
        got = ref.clone()
        hot = flat
    got[hot[:need, 0], hot[:need, 1]] = Tm - 1.0
    d, a, back = judge(got, ref, 5.0, 0.02, Tm)
    assert d <= 5.0 and a >= 0.03 and back is True
    got = ref.clone()
    got[0, 0] = float("nan")
    assert judge(got, ref, 5.0, 0.02, Tm)[2] is True
