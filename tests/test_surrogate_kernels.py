# SPDX-License-Identifier: 0BSD
"""Tensor-core layers of the learned super-stepper (lpbf_b200_sg_conv,
lpbf_b200_sg_gemm_bt) against the FP64 numpy restatement in
oracle/surrogate_ref.py, on the same bf16-rounded operands.  Tolerance: the
fp32-accumulated result is rounded to bf16 on output (relative step 2^-8),
so outputs agree within 1e-2 relative to the largest output magnitude."""
import ctypes

import numpy as np
import pytest

from oracle import surrogate_ref as R

pytestmark = pytest.mark.gpu


def _bf16(a):
    import torch
    return torch.tensor(np.asarray(a, dtype=np.float32)).to(torch.bfloat16)


def _np(t):
    import torch
    return t.float().cpu().numpy().astype(np.float64) if t.dtype == torch.bfloat16 \
        else t.cpu().numpy().astype(np.float64)


def _conv(kind, x, wp, bias=None, pre_in=None, want_pre=False, out_fp32=False):
    import torch
    from hedgehog_lpbf_b200 import _lib
    L = _lib.lib()
    dev = torch.device("cuda:0")
    B, H, W = x.shape[:3]
    xd = x.to(dev).contiguous()
    wd = wp.to(dev).contiguous()
    bd = torch.tensor(bias, dtype=torch.float32, device=dev) if bias is not None else None
    pid = pre_in.to(dev).contiguous() if pre_in is not None else None
    if out_fp32:
        out = torch.zeros((B, H, W), dtype=torch.float32, device=dev)
    else:
        out = torch.zeros((B, H, W, 32), dtype=torch.bfloat16, device=dev)
    pre = torch.zeros((B, H, W, 32), dtype=torch.bfloat16, device=dev) if want_pre else None
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    a = _lib.SgConvArgs(x=xd.data_ptr(), w=wd.data_ptr(), bias=bd.data_ptr() if bd is not None else None,
                        pre_in=pid.data_ptr() if pid is not None else None,
                        pre_out=pre.data_ptr() if pre is not None else None, out=out.data_ptr(),
                        batch=B, height=H, width=W, err=err.data_ptr())
    st = L.lpbf_b200_sg_conv(kind, ctypes.byref(a), torch.cuda.current_stream().cuda_stream)
    assert st == 0, L.lpbf_b200_status_string(st)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    return out, pre


def _close(got, ref, rtol=1e-2):
    scale = max(np.max(np.abs(ref)), 1e-6)
    assert np.max(np.abs(got - ref)) <= rtol * scale, (np.max(np.abs(got - ref)), scale)


def test_tile_product_on_tensor_cores(gpu):
    import torch
    from hedgehog_lpbf_b200 import _lib
    L = _lib.lib()
    rng = np.random.default_rng(0)
    for n in (32, 16):
        A = _bf16(rng.normal(size=(128, 288)))
        B = _bf16(rng.normal(size=(n, 288)))
        C = torch.zeros((128, n), dtype=torch.float32, device="cuda:0")
        err = torch.zeros(1, dtype=torch.int32, device="cuda:0")
        Ad, Bd = A.cuda(), B.cuda()
        assert L.lpbf_b200_sg_gemm_bt(Ad.data_ptr(), Bd.data_ptr(), C.data_ptr(), n, 288,
                                      err.data_ptr(), None) == 0
        torch.cuda.synchronize()
        assert int(err.item()) == 0
        ref = _np(A) @ _np(B).T
        assert np.max(np.abs(_np(C) - ref)) <= 1e-4 * np.max(np.abs(ref))


@pytest.mark.parametrize("B,H,W", [(1, 3, 128), (2, 5, 200), (1, 2, 300)])
def test_forward_layers(gpu, B, H, W):
    rng = np.random.default_rng(1)
    ps = R.init_params(3)
    x4 = _bf16(rng.normal(size=(B, H, W, 4)))
    # input layer 4 -> 32
    w, b = ps[0]
    b = rng.normal(size=32) * 0.1
    act, pre = _conv(0, x4, _bf16(R.pack(w, k_pad=64)), bias=b, want_pre=True)
    ref_pre = R.conv3x3(_np(x4), _np(_bf16(w.reshape(32, -1))).reshape(w.shape), b)
    _close(_np(pre), ref_pre)
    _close(_np(act), R.gelu(_np(pre)))
    # hidden 32 -> 32 on the (bf16) activations
    w, _ = ps[1]
    wq = _np(_bf16(w.reshape(32, -1))).reshape(w.shape)
    act2, pre2 = _conv(1, act, _bf16(R.pack(w)), bias=b, want_pre=True)
    _close(_np(pre2), R.conv3x3(_np(act), wq, b))
    # output 32 -> 1
    w, _ = ps[4]
    wq = _np(_bf16(w.reshape(1, -1))).reshape(w.shape)
    y, _ = _conv(2, act2, _bf16(R.pack(w, n_pad=16)), bias=np.array([0.25]), out_fp32=True)
    _close(_np(y), R.conv3x3(_np(act2), wq, np.array([0.25]))[..., 0], rtol=2e-3)


def test_input_gradient_layers(gpu):
    rng = np.random.default_rng(2)
    B, H, W = 2, 4, 170
    ps = R.init_params(5)
    pre_prev = _bf16(rng.normal(size=(B, H, W, 32)))
    # output layer: upstream gradient has one channel
    g5 = _bf16(rng.normal(size=(B, H, W, 1)))
    w5 = ps[4][0]
    wt = R.flip_transpose(w5)                      # [32, 9, 1]
    out, _ = _conv(3, g5, _bf16(R.pack(wt, k_pad=64)), pre_in=pre_prev)
    wq = _np(_bf16(wt.reshape(32, -1))).reshape(wt.shape)
    ref = R.conv3x3(_np(g5), wq) * R.gelu_grad(_np(pre_prev))
    _close(_np(out), ref)
    # hidden layer
    g = _bf16(rng.normal(size=(B, H, W, 32)))
    w = ps[2][0]
    wt = R.flip_transpose(w)
    out, _ = _conv(4, g, _bf16(R.pack(wt)), pre_in=pre_prev)
    wq = _np(_bf16(wt.reshape(32, -1))).reshape(wt.shape)
    ref = R.conv3x3(_np(g), wq) * R.gelu_grad(_np(pre_prev))
    _close(_np(out), ref)
    # the flipped-transposed weights are the adjoint of the forward conv
    x = rng.normal(size=(1, 3, 7, 32))
    gg = rng.normal(size=(1, 3, 7, 32))
    lhs = np.sum(R.conv3x3(x, w) * gg)
    rhs = np.sum(x * R.conv3x3_input_grad(gg, w))
    assert abs(lhs - rhs) <= 1e-9 * abs(lhs)


def _rand_net(seed, out_std=0.3):
    ps = R.init_params(seed)
    rng = np.random.default_rng(seed + 100)
    ps = [(w, rng.normal(0, 0.05, b.shape)) for w, b in ps]
    w5, b5 = ps[4]
    ps[4] = (w5 * out_std / 0.1 * 10, b5)
    return ps


def _bf16_params(ps):
    return [(_np(_bf16(w.reshape(w.shape[0], -1))).reshape(w.shape), b) for w, b in ps]


@pytest.mark.parametrize("B,H,W,form", [(2, 6, 150, 0), (2, 6, 150, 1), (2, 70, 260, 0)])
def test_weight_gradients_match_fp64_backward(gpu, B, H, W, form):
    """Gradient check: the GPU's loss and per-layer gradients (bf16 operands,
    fp32 accumulation) against the FP64 backward pass of oracle/surrogate_ref
    on the same bf16-rounded inputs and weights, with the row-streaming
    layers and weight gradients (form 0; 70 rows: three runs of rows per
    column tile) and the tap-tile ones (form 1)."""
    import torch
    from hedgehog_lpbf_b200 import _lib
    from hedgehog_lpbf_b200.surrogate import Net, unflatten
    L = _lib.lib()
    rng = np.random.default_rng(7)
    ps = _rand_net(3)
    x4 = _bf16(rng.normal(size=(B, H, W, 4)))
    tgt = rng.normal(size=(B, H, W)).astype(np.float32)
    net = Net(ps, device="cuda:0")
    try:
        assert L.lpbf_b200_sg_set_form(form) == 0
        loss = net.gradients(x4.cuda(), torch.tensor(tgt, device="cuda:0"))
        torch.cuda.synchronize()
    finally:
        L.lpbf_b200_sg_set_form(0)
    assert net.error_word() == 0
    g_gpu = unflatten(net.grads_vector())
    loss_ref, g_ref = R.loss_and_grads(_bf16_params(ps), _np(x4), tgt.astype(np.float64))
    assert abs(float(loss.item()) - loss_ref) <= 1e-2 * loss_ref
    for li in range(5):
        for part in (0, 1):
            a, b = g_gpu[li][part].ravel(), g_ref[li][part].ravel()
            rel = np.linalg.norm(a - b) / np.linalg.norm(b)
            cos = a @ b / (np.linalg.norm(a) * np.linalg.norm(b))
            assert rel < 3e-2 and cos > 0.999, (li, part, rel, cos)


def test_adamw_step_matches_reference(gpu):
    import torch
    from hedgehog_lpbf_b200.surrogate import Net
    rng = np.random.default_rng(8)
    ps = _rand_net(4)
    x4 = _bf16(rng.normal(size=(1, 4, 130, 4)))
    tgt = torch.tensor(rng.normal(size=(1, 4, 130)).astype(np.float32), device="cuda:0")
    net = Net(ps, device="cuda:0")
    p0 = net.params_vector().astype(np.float64)
    net.train_step(x4.cuda(), tgt, lr=1e-3, weight_decay=0.01)
    torch.cuda.synchronize()
    g = net.grads_vector().astype(np.float64)
    p1 = net.params_vector().astype(np.float64)
    ref, _, _ = R.adamw(p0, g, np.zeros_like(g), np.zeros_like(g), 1, lr=1e-3, wd=0.01)
    assert np.max(np.abs(p1 - ref)) <= 1e-6 * max(1.0, np.max(np.abs(ref)))
    # a second step moves on from the stored moments
    net.train_step(x4.cuda(), tgt, lr=1e-3, weight_decay=0.01)
    torch.cuda.synchronize()
    assert not np.array_equal(net.params_vector(), p1.astype(np.float32))


def test_features_and_apply(gpu):
    import torch
    from hedgehog_lpbf_b200 import params as P
    from hedgehog_lpbf_b200 import plan as PL
    from hedgehog_lpbf_b200.surrogate import features, apply, target, STEPS
    mat, pr = P.benchmark_material_process()
    dom = P.square_domain(200)
    k = P.make_const(mat, pr, dom, P.dt_fraction(mat, dom))
    plan = PL.raster_for_steps(dom, k.dt, 64, V=1.0, hatch=100e-6, n_tracks=2)
    rng = np.random.default_rng(3)
    T = 300.0 + rng.uniform(0, 1500, size=(200, 200))
    Td = torch.tensor(T, device="cuda:0")
    x4 = features(Td, k, plan).float().cpu().numpy()
    yy, xx = np.meshgrid(np.arange(200) * k.dy, np.arange(200) * k.dx, indexing="ij")
    S = np.zeros_like(T)
    for s in range(STEPS):
        cs = k.dt * (plan["q_scale"][s] * k.peak_S) / (k.rho_cp * k.h)
        r2 = (xx - plan["x_l"][s]) ** 2 + (yy - plan["y_l"][s]) ** 2
        S += cs * np.exp(-2.0 * r2 * k.inv_r0_sq)
    ref = np.stack([(T - k.Tamb) / 1000.0, S / 1000.0,
                    np.clip((xx - plan["x_l"][8]) / 100e-6, -8, 8),
                    np.clip((yy - plan["y_l"][8]) / 100e-6, -8, 8)], axis=-1)
    assert np.max(np.abs(x4 - ref)) <= 1e-2 * np.max(np.abs(ref))
    y = torch.tensor(rng.normal(size=(200, 200)).astype(np.float32), device="cuda:0")
    T1 = Td.clone()
    apply(T1, y)
    assert np.allclose(T1.cpu().numpy(), T + 100.0 * y.cpu().numpy().astype(np.float64))
    t = target(Td, T1).cpu().numpy()
    assert np.allclose(t, y.cpu().numpy(), rtol=1e-5, atol=1e-5)


@pytest.mark.parametrize("B,H,W", [(2, 70, 260), (1, 33, 128), (3, 1, 90), (1, 4, 131)])
def test_conv_forms_agree(gpu, B, H, W):
    """The row-streaming, tap-tile and plain forms against the FP64
    restatement on images with ragged row runs (H not a multiple of 32),
    ragged column tiles and an odd width (the input layer's row form needs
    an even one and falls back); the 32-channel forms agree bit for bit."""
    from hedgehog_lpbf_b200 import _lib
    L = _lib.lib()
    rng = np.random.default_rng(7)
    ps = R.init_params(11)
    x4 = _bf16(rng.normal(size=(B, H, W, 4)))
    act = _bf16(rng.normal(size=(B, H, W, 32)))
    pre_prev = _bf16(rng.normal(size=(B, H, W, 32)))
    b = rng.normal(size=32) * 0.1
    w0, w1, w4 = ps[0][0], ps[1][0], ps[4][0]
    w0q = _np(_bf16(w0.reshape(32, -1))).reshape(w0.shape)
    w1q = _np(_bf16(w1.reshape(32, -1))).reshape(w1.shape)
    w4q = _np(_bf16(w4.reshape(1, -1))).reshape(w4.shape)
    wt = R.flip_transpose(ps[2][0])
    wtq = _np(_bf16(wt.reshape(32, -1))).reshape(wt.shape)
    ref_in = R.conv3x3(_np(x4), w0q, b)
    ref_pre = R.conv3x3(_np(act), w1q, b)
    ref_y = R.conv3x3(_np(act), w4q, np.array([0.25]))[..., 0]
    ref_dx = R.conv3x3(_np(act), wtq) * R.gelu_grad(_np(pre_prev))
    got = {}
    try:
        for form in (0, 1, 2):
            assert L.lpbf_b200_sg_set_form(form) == 0
            act0, pre0 = _conv(0, x4, _bf16(R.pack(w0, k_pad=64)), bias=b, want_pre=True)
            assert L.lpbf_b200_sg_form_used() == (2 if form or W % 2 else 0)
            _close(_np(pre0), ref_in)
            _close(_np(act0), R.gelu(_np(pre0)))
            act2, pre2 = _conv(1, act, _bf16(R.pack(w1)), bias=b, want_pre=True)
            y, _ = _conv(2, act, _bf16(R.pack(w4, n_pad=16)), bias=np.array([0.25]),
                         out_fp32=True)
            dx, _ = _conv(4, act, _bf16(R.pack(wt)), pre_in=pre_prev)
            assert L.lpbf_b200_sg_form_used() == form
            _close(_np(pre2), ref_pre)
            _close(_np(act2), R.gelu(_np(pre2)))
            _close(_np(y), ref_y, rtol=2e-3)
            _close(_np(dx), ref_dx)
            got[form] = [_np(t) for t in (pre2, act2, y, dx)]
    finally:
        L.lpbf_b200_sg_set_form(0)
    # same operands, same tap order: the 32-channel forms agree bit for bit
    for form in (1, 2):
        for a, c in zip(got[0], got[form]):
            assert np.array_equal(a, c)
    assert L.lpbf_b200_sg_set_form(3) != 0


def test_weight_gradient_forms_agree_at_size(gpu):
    """576 row runs (more than one per CTA of the row-streaming weight
    gradient): its gradients against the tap-tile form's on 2.4 M pixels
    (the same operands; fp32 sums in other orders)."""
    import torch
    from hedgehog_lpbf_b200 import _lib
    from hedgehog_lpbf_b200.surrogate import Net, unflatten
    L = _lib.lib()
    rng = np.random.default_rng(9)
    B, H, W = 24, 256, 384
    ps = _rand_net(6)
    x4 = _bf16(rng.normal(size=(B, H, W, 4))).cuda()
    tgt = torch.tensor(rng.normal(size=(B, H, W)).astype(np.float32), device="cuda:0")
    grads = {}
    try:
        for form in (0, 1):
            assert L.lpbf_b200_sg_set_form(form) == 0
            net = Net(ps, device="cuda:0")
            net.gradients(x4, tgt)
            torch.cuda.synchronize()
            assert net.error_word() == 0
            grads[form] = unflatten(net.grads_vector())
            del net
    finally:
        L.lpbf_b200_sg_set_form(0)
    for li in range(5):
        for part in (0, 1):
            a, b = grads[0][li][part].ravel(), grads[1][li][part].ravel()
            rel = np.linalg.norm(a - b) / np.linalg.norm(b)
            cos = a @ b / (np.linalg.norm(a) * np.linalg.norm(b))
            assert rel < 1e-2 and cos > 0.9999, (li, part, rel, cos)
