# SPDX-License-Identifier: 0BSD
"""Python host of the learned super-stepper (lpbf_b200_sg_* in
include/lpbf_b200.h): the network blob, forward, gradients, AdamW training
steps and the features of a field.  Every computation runs in
liblpbf_b200.so (tcgen05 tensor-core layers); torch only holds device memory.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from . import _lib
from .params import StepConst
from .plan import TICK_DTYPE
from .solver import _stream_handle

CH = (4, 32, 32, 32, 32, 1)
STEPS = 16                   # time steps per super-step (LPBF_SG_STEPS)
T_SCALE, S_SCALE, DT_SCALE, POS_SCALE = 1000.0, 1000.0, 100.0, 100e-6


def layer_shapes():
    return [((CH[i + 1], 9, CH[i]), (CH[i + 1],)) for i in range(5)]


def flatten(params) -> np.ndarray:
    """[(W [co, 9, ci], b [co]), ...] -> the blob's parameter vector."""
    return np.concatenate([np.concatenate([np.asarray(w).ravel(), np.asarray(b).ravel()])
                           for w, b in params]).astype(np.float32)


def unflatten(v: np.ndarray):
    out, o = [], 0
    for ws, bs in layer_shapes():
        nw, nb = int(np.prod(ws)), bs[0]
        out.append((v[o:o + nw].reshape(ws).astype(np.float64),
                    v[o + nw:o + nw + nb].astype(np.float64)))
        o += nw + nb
    return out


def init_params(seed: int = 0):
    """He-normal hidden layers, a small output layer, zero biases."""
    rng = np.random.default_rng(seed)
    ps = []
    for i, ((co, _, ci), _) in enumerate(layer_shapes()):
        std = math.sqrt(2.0 / (9 * ci)) if i < 4 else 0.1 * math.sqrt(1.0 / (9 * ci))
        ps.append((rng.normal(0.0, std, (co, 9, ci)), np.zeros(co)))
    return ps


class Net:
    """The network blob on one device with its activation workspace."""

    def __init__(self, params=None, device: torch.device | str | None = None, seed: int = 0):
        self.lib = _lib.lib()
        self.device = torch.device(device) if device is not None else torch.device("cuda")
        self.np = self.lib.lpbf_b200_sg_param_count()
        self.blob = torch.zeros(self.lib.lpbf_b200_sg_net_bytes(), dtype=torch.uint8,
                                device=self.device)
        self.err = torch.zeros(1, dtype=torch.int32, device=self.device)
        self.loss = torch.zeros(1, dtype=torch.float32, device=self.device)
        self._work = None
        self._work_key = None
        self.step = 0
        self.set_params(params if params is not None else init_params(seed))

    # -- parameters ----------------------------------------------------------
    def set_params(self, params) -> None:
        v = flatten(params) if not isinstance(params, np.ndarray) else params.astype(np.float32)
        assert v.size == self.np
        t = torch.tensor(v, device=self.device)
        with torch.cuda.device(self.device):
            _lib.check(self.lib.lpbf_b200_sg_net_set(self.blob.data_ptr(), t.data_ptr(),
                                                     _stream_handle(None)), "sg_net_set")
        torch.cuda.synchronize(self.device)
        self.step = 0

    def params_vector(self) -> np.ndarray:
        out = torch.empty(self.np, dtype=torch.float32, device=self.device)
        with torch.cuda.device(self.device):
            _lib.check(self.lib.lpbf_b200_sg_net_get(self.blob.data_ptr(), out.data_ptr(), None,
                                                     _stream_handle(None)), "sg_net_get")
        return out.cpu().numpy()

    def grads_vector(self) -> np.ndarray:
        out = torch.empty(self.np, dtype=torch.float32, device=self.device)
        with torch.cuda.device(self.device):
            _lib.check(self.lib.lpbf_b200_sg_net_get(self.blob.data_ptr(), None, out.data_ptr(),
                                                     _stream_handle(None)), "sg_net_get")
        return out.cpu().numpy()

    # -- workspace -----------------------------------------------------------
    def work(self, B, H, W, train):
        key = (B, H, W, bool(train))
        need = self.lib.lpbf_b200_sg_work_bytes(B, H, W, int(train))
        if self._work is None or self._work.numel() < need:
            self._work = torch.empty(need, dtype=torch.uint8, device=self.device)
        self._work_key = key
        return self._work

    # -- compute -------------------------------------------------------------
    def forward(self, x4: torch.Tensor, y: torch.Tensor | None = None) -> torch.Tensor:
        """x4: bf16 [B, H, W, 4] -> y fp32 [B, H, W]."""
        B, H, W = x4.shape[:3]
        if y is None:
            y = torch.empty((B, H, W), dtype=torch.float32, device=self.device)
        w = self.work(B, H, W, False)
        with torch.cuda.device(self.device):
            _lib.check(self.lib.lpbf_b200_sg_forward(
                self.blob.data_ptr(), x4.data_ptr(), y.data_ptr(), B, H, W, w.data_ptr(),
                w.numel(), self.err.data_ptr(), _stream_handle(None)), "sg_forward")
        return y

    def gradients(self, x4, target):
        B, H, W = x4.shape[:3]
        w = self.work(B, H, W, True)
        with torch.cuda.device(self.device):
            _lib.check(self.lib.lpbf_b200_sg_gradients(
                self.blob.data_ptr(), x4.data_ptr(), target.data_ptr(), B, H, W, w.data_ptr(),
                w.numel(), self.loss.data_ptr(), self.err.data_ptr(), _stream_handle(None)),
                "sg_gradients")
        return self.loss

    def train_step(self, x4, target, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8,
                   weight_decay=0.01):
        B, H, W = x4.shape[:3]
        w = self.work(B, H, W, True)
        self.step += 1
        h = _lib.SgHyper(lr=lr, beta1=beta1, beta2=beta2, eps=eps, weight_decay=weight_decay,
                         step=self.step)
        with torch.cuda.device(self.device):
            _lib.check(self.lib.lpbf_b200_sg_train_step(
                self.blob.data_ptr(), x4.data_ptr(), target.data_ptr(), B, H, W, ctypes.byref(h),
                w.data_ptr(), w.numel(), self.loss.data_ptr(), self.err.data_ptr(),
                _stream_handle(None)), "sg_train_step")
        return self.loss

    def error_word(self) -> int:
        return int(self.err.item())


def features(T: torch.Tensor, k: StepConst, plan: np.ndarray, out: torch.Tensor | None = None):
    """Network inputs (bf16 [ny, nx, 4]) of field T (fp64 [ny, nx]) before
    plan[:STEPS]."""
    L = _lib.lib()
    ny, nx = T.shape
    if out is None:
        out = torch.empty((ny, nx, 4), dtype=torch.bfloat16, device=T.device)
    p = np.ascontiguousarray(plan[:STEPS], dtype=TICK_DTYPE)
    assert len(p) == STEPS
    with torch.cuda.device(T.device):
        _lib.check(L.lpbf_b200_sg_features(T.data_ptr(), ctypes.byref(k), p.ctypes.data,
                                           out.data_ptr(), _stream_handle(None)), "sg_features")
    return out


def target(T0: torch.Tensor, T1: torch.Tensor, out: torch.Tensor | None = None):
    L = _lib.lib()
    if out is None:
        out = torch.empty(T0.shape, dtype=torch.float32, device=T0.device)
    with torch.cuda.device(T0.device):
        _lib.check(L.lpbf_b200_sg_target(T0.data_ptr(), T1.data_ptr(), out.data_ptr(),
                                         T0.numel(), _stream_handle(None)), "sg_target")
    return out


def apply(T: torch.Tensor, y: torch.Tensor) -> None:
    L = _lib.lib()
    with torch.cuda.device(T.device):
        _lib.check(L.lpbf_b200_sg_apply(T.data_ptr(), y.data_ptr(), T.numel(),
                                        _stream_handle(None)), "sg_apply")
