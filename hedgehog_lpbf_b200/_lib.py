# SPDX-License-Identifier: 0BSD
"""ctypes binding of liblpbf_b200.so (the C-ABI of include/lpbf_kernels.hpp
and include/lpbf_b200.h).

The library is built in-tree by ``hedgehog_lpbf_b200.build``.  There is no
fallback: if the library cannot be built or loaded, ``lib()`` raises.
"""
from __future__ import annotations

import ctypes
import os
import threading

from . import build as _build
from .params import Partial, StepConst, Tick

_lock = threading.Lock()
_lib = None

LPBF_OK = 0
_vp = ctypes.c_void_p
_dp = ctypes.POINTER(ctypes.c_double)


class Opts(ctypes.Structure):
    """lpbf_b200_opts (include/lpbf_b200.h)."""
    _fields_ = [("phys", ctypes.c_int), ("bc", ctypes.c_int), ("T_edge", ctypes.c_double),
                ("Tm", ctypes.c_double), ("depth", ctypes.c_int), ("rows", ctypes.c_int)]


class Rows(ctypes.Structure):
    """lpbf_b200_rows (include/lpbf_b200.h): a row strip of a larger field."""
    _fields_ = [("row0", ctypes.c_int), ("global_ny", ctypes.c_int), ("lo", ctypes.c_int),
                ("hi", ctypes.c_int)]


class Scenario(ctypes.Structure):
    """lpbf_b200_scenario (include/lpbf_b200.h)."""
    _fields_ = [("k", ctypes.POINTER(StepConst)), ("plan", _vp), ("T_a", _vp), ("T_b", _vp),
                ("ring", _vp), ("bc", ctypes.c_int), ("T_edge", ctypes.c_double),
                ("Tm", ctypes.c_double)]


class BatchOpts(ctypes.Structure):
    """lpbf_b200_batch_opts (include/lpbf_b200.h)."""
    _fields_ = [("depth", ctypes.c_int), ("ctas_per_sm", ctypes.c_int),
                ("rows", ctypes.c_int * 4), ("staging", ctypes.c_int)]


class SgConvArgs(ctypes.Structure):
    """lpbf_b200_sg_conv_args (include/lpbf_b200.h)."""
    _fields_ = [("x", _vp), ("w", _vp), ("bias", _vp), ("pre_in", _vp), ("pre_out", _vp),
                ("out", _vp), ("batch", ctypes.c_int), ("height", ctypes.c_int),
                ("width", ctypes.c_int), ("err", _vp)]


class SgHyper(ctypes.Structure):
    """lpbf_b200_sg_hyper (include/lpbf_b200.h)."""
    _fields_ = [("lr", ctypes.c_float), ("beta1", ctypes.c_float), ("beta2", ctypes.c_float),
                ("eps", ctypes.c_float), ("weight_decay", ctypes.c_float), ("step", ctypes.c_int)]


_sp = ctypes.POINTER(Scenario)
_bop = ctypes.POINTER(BatchOpts)

# name -> (restype, argtypes); every symbol the headers in include/ declare.
SIGNATURES = {
    # include/lpbf_kernels.hpp (reference drop-in)
    "lpbf_launch_step": (None, [_vp, _vp, ctypes.POINTER(StepConst), ctypes.c_int, _vp]),
    "lpbf_launch_reduce": (None, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_double, _vp,
                                  ctypes.c_int, _vp]),
    "lpbf_launch_step_reduce": (None, [_vp, _vp, ctypes.POINTER(StepConst), ctypes.c_int,
                                       ctypes.c_double, _vp, _vp]),
    "lpbf_launch_reduce_finalize": (None, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp,
                                           _vp]),
    "lpbf_launch_extract_col": (None, [_vp, ctypes.c_int, ctypes.c_int, _vp, _vp, _vp]),
    # include/lpbf_b200.h
    "lpbf_b200_version": (ctypes.c_int, []),
    "lpbf_b200_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "lpbf_b200_workspace_bytes": (ctypes.c_size_t, []),
    "lpbf_b200_workspace_init": (ctypes.c_int, [_vp, ctypes.c_size_t, _vp]),
    "lpbf_b200_advance": (ctypes.c_int, [_vp, _vp, ctypes.POINTER(StepConst), _vp, ctypes.c_int,
                                         ctypes.POINTER(Opts), _vp, _vp, ctypes.c_size_t, _vp,
                                         ctypes.POINTER(ctypes.c_int)]),
    "lpbf_b200_advance_launches": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                  ctypes.POINTER(Opts)]),
    "lpbf_b200_advance_rows": (ctypes.c_int, [_vp, _vp, ctypes.POINTER(StepConst), _vp,
                                              ctypes.c_int, ctypes.POINTER(Opts),
                                              ctypes.POINTER(Rows), _vp, _vp, ctypes.c_size_t,
                                              _vp]),
    "lpbf_b200_read_error": (ctypes.c_int, [_vp, _vp, ctypes.POINTER(ctypes.c_uint)]),
    "lpbf_b200_advance_f32k": (ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.POINTER(StepConst), _vp,
                                              ctypes.c_int, ctypes.POINTER(Opts), _vp, _vp,
                                              ctypes.c_size_t, _vp, ctypes.POINTER(ctypes.c_int)]),
    "lpbf_b200_f32k_split": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_size_t, _vp]),
    "lpbf_b200_f32k_join": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_size_t, _vp]),
    "lpbf_b200_advance_f32": (ctypes.c_int, [_vp, _vp, ctypes.POINTER(StepConst), _vp,
                                             ctypes.c_int, ctypes.POINTER(Opts), _vp, _vp,
                                             ctypes.c_size_t, _vp, ctypes.POINTER(ctypes.c_int)]),
    "lpbf_b200_advance_noalloc": (ctypes.c_int, [_vp, _vp, ctypes.POINTER(StepConst), _vp,
                                                 ctypes.c_int, ctypes.POINTER(Opts), _vp, _vp,
                                                 ctypes.POINTER(ctypes.c_int),
                                                 ctypes.POINTER(ctypes.c_uint)]),
    "lpbf_b200_batch_size_class": (ctypes.c_int, [ctypes.c_int, ctypes.c_int]),
    "lpbf_b200_batch_workspace_bytes": (ctypes.c_size_t, [_sp, ctypes.c_int, ctypes.c_int, _bop]),
    "lpbf_b200_batch_create": (ctypes.c_int, [_sp, ctypes.c_int, ctypes.c_int, _bop, _vp,
                                              ctypes.c_size_t, _vp, ctypes.POINTER(_vp)]),
    "lpbf_b200_batch_run": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp]),
    "lpbf_b200_batch_capture": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int]),
    "lpbf_b200_batch_run_wsub": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _vp, _vp, _vp]),
    "lpbf_b200_batch_result_in_b": (ctypes.c_int, [_vp]),
    "lpbf_b200_batch_launches": (ctypes.c_int, [_vp, ctypes.c_int]),
    "lpbf_b200_batch_tasks": (ctypes.c_int, [_vp]),
    "lpbf_b200_batch_scenario_rows": (ctypes.c_int, [_vp, ctypes.c_int]),
    "lpbf_b200_batch_read_error": (ctypes.c_int, [_vp, _vp, ctypes.POINTER(ctypes.c_uint)]),
    "lpbf_b200_batch_destroy": (None, [_vp]),
    "lpbf_b200_batch_autotune": (ctypes.c_int, [_sp, ctypes.c_int, ctypes.c_int, ctypes.c_char_p,
                                                ctypes.c_int, _bop]),
    "lpbf_b200_batch_tune_key": (ctypes.c_int, [_sp, ctypes.c_int, ctypes.c_char_p,
                                                ctypes.c_size_t]),
    "lpbf_b200_tune_cache_get": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, _bop]),
    "lpbf_b200_tune_cache_put": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, _bop,
                                                ctypes.c_double]),
    "lpbf_b200_sg_conv": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(SgConvArgs), _vp]),
    "lpbf_b200_sg_gemm_bt": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int, ctypes.c_int, _vp, _vp]),
    "lpbf_b200_sg_set_form": (ctypes.c_int, [ctypes.c_int]),
    "lpbf_b200_sg_form_used": (ctypes.c_int, []),
    "lpbf_b200_sg_param_count": (ctypes.c_int, []),
    "lpbf_b200_sg_net_bytes": (ctypes.c_size_t, []),
    "lpbf_b200_sg_work_bytes": (ctypes.c_size_t, [ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                  ctypes.c_int]),
    "lpbf_b200_sg_net_set": (ctypes.c_int, [_vp, _vp, _vp]),
    "lpbf_b200_sg_net_get": (ctypes.c_int, [_vp, _vp, _vp, _vp]),
    "lpbf_b200_sg_forward": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int, ctypes.c_int,
                                            ctypes.c_int, _vp, ctypes.c_size_t, _vp, _vp]),
    "lpbf_b200_sg_gradients": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int, ctypes.c_int,
                                              ctypes.c_int, _vp, ctypes.c_size_t, _vp, _vp, _vp]),
    "lpbf_b200_sg_adamw": (ctypes.c_int, [_vp, ctypes.POINTER(SgHyper), _vp]),
    "lpbf_b200_sg_train_step": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int, ctypes.c_int,
                                               ctypes.c_int, ctypes.POINTER(SgHyper), _vp,
                                               ctypes.c_size_t, _vp, _vp, _vp]),
    "lpbf_b200_sg_features": (ctypes.c_int, [_vp, ctypes.POINTER(StepConst), _vp, _vp, _vp]),
    "lpbf_b200_sg_apply": (ctypes.c_int, [_vp, _vp, ctypes.c_longlong, _vp]),
    "lpbf_b200_sg_target": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_longlong, _vp]),
}


def lib_path() -> str:
    return _build.LIB


def lib(build_if_needed: bool = True):
    """Load liblpbf_b200.so, building it first if it is missing or stale."""
    global _lib
    with _lock:
        if _lib is None:
            if build_if_needed and (_build.stale() and _can_build()):
                _build.build()
            if not os.path.exists(_build.LIB):
                raise RuntimeError(f"{_build.LIB} is missing and could not be built")
            L = ctypes.CDLL(_build.LIB)
            for name, (res, args) in SIGNATURES.items():
                f = getattr(L, name)
                f.restype = res
                f.argtypes = args
            _lib = L
    return _lib


def _can_build() -> bool:
    try:
        _build.nvcc()
        return True
    except RuntimeError:
        return False


def check(status: int, what: str = "liblpbf_b200") -> None:
    if status != LPBF_OK:
        msg = lib().lpbf_b200_status_string(status).decode()
        raise RuntimeError(f"{what}: status {status} ({msg})")


__all__ = ["lib", "lib_path", "check", "Opts", "Scenario", "BatchOpts", "SIGNATURES", "StepConst",
           "Partial", "Tick"]
