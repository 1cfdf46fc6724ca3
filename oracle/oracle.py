# SPDX-License-Identifier: 0BSD
"""ORACLE -- test infrastructure only.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may
import this module, and only as the checker.  It wraps:

* ``oracle/_build/liblpbf_oracle.so`` -- the plain-C restatement of the
  reference's CPU step (oracle/lpbf_oracle.c), built from source with
  ``make -C oracle`` on first use (gcc is on every machine this runs on);
* ``oracle/_ref/*.so`` -- the reference's own CPU code compiled from the
  reference tree (``make -C oracle ref``).  Those exist only where the
  reference tree was available at build time; ``have_reference()`` says so.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_BUILD = os.path.join(HERE, "_build")
_REF = os.path.join(HERE, "_ref")
_lock = threading.Lock()
_lib = None
_ref = {}


class OracleStepConst(ctypes.Structure):
    """C mirror of the reference StepConst (lpbf_step_const.hpp:19-29)."""
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int),
        ("dx", ctypes.c_double), ("dy", ctypes.c_double),
        ("inv_dx2", ctypes.c_double), ("inv_dy2", ctypes.c_double),
        ("inv_r0_sq", ctypes.c_double),
        ("alpha", ctypes.c_double), ("K", ctypes.c_double), ("rho", ctypes.c_double),
        ("cp", ctypes.c_double), ("rho_cp", ctypes.c_double), ("inv_h", ctypes.c_double),
        ("h", ctypes.c_double), ("dt", ctypes.c_double),
        ("peak_S", ctypes.c_double), ("eta", ctypes.c_double), ("P", ctypes.c_double),
        ("hConv", ctypes.c_double), ("Tamb", ctypes.c_double), ("Tsub", ctypes.c_double),
        ("dSub", ctypes.c_double), ("eps", ctypes.c_double),
        ("radiation", ctypes.c_bool), ("kmult", ctypes.c_double),
        ("x_l", ctypes.c_double), ("y_l", ctypes.c_double), ("q_scale", ctypes.c_double),
    ]


class OraclePartial(ctypes.Structure):
    _fields_ = [("tmax", ctypes.c_double), ("arg", ctypes.c_longlong),
                ("ymin", ctypes.c_int), ("ymax", ctypes.c_int)]


class OracleMeasure(ctypes.Structure):
    _fields_ = [("peak_T", ctypes.c_double), ("x_hot", ctypes.c_int),
                ("W_um", ctypes.c_double), ("W_sub_um", ctypes.c_double)]


PARTIAL_DTYPE = np.dtype({"names": ["tmax", "arg", "ymin", "ymax"],
                          "formats": [np.float64, np.int64, np.int32, np.int32],
                          "offsets": [0, 8, 16, 20], "itemsize": 24})

_dp = ctypes.POINTER(ctypes.c_double)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def lib():
    """The C restatement, built on first use."""
    global _lib
    with _lock:
        if _lib is None:
            so = os.path.join(_BUILD, "liblpbf_oracle.so")
            src = os.path.join(HERE, "lpbf_oracle.c")
            if not os.path.exists(so) or os.path.getmtime(so) < os.path.getmtime(src):
                subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
            L = ctypes.CDLL(so)
            sc = ctypes.POINTER(OracleStepConst)
            L.oracle_step.argtypes = [_dp, _dp, sc, ctypes.c_int, ctypes.c_int, ctypes.c_double]
            L.oracle_reduce.argtypes = [_dp, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                        ctypes.POINTER(OraclePartial)]
            L.oracle_measure.argtypes = [_dp, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                         ctypes.c_double, ctypes.POINTER(OracleMeasure)]
            L.oracle_w_sub.argtypes = [_dp, ctypes.c_int, ctypes.c_double, ctypes.c_double]
            L.oracle_w_sub.restype = ctypes.c_double
            L.oracle_run.argtypes = [_dp, _dp, sc, _dp, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                     ctypes.c_void_p]
            L.oracle_run.restype = ctypes.c_int
            L.oracle_run_quiet.argtypes = [_dp, _dp, sc, _dp, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_double, ctypes.c_double, ctypes.c_void_p,
                                           ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
            L.oracle_run_quiet.restype = ctypes.c_int
            for f in ("oracle_k_of", "oracle_cp_of", "oracle_cp_eff"):
                getattr(L, f).argtypes = [ctypes.c_double]
                getattr(L, f).restype = ctypes.c_double
            for f in ("oracle_k_enh", "oracle_k_eff"):
                getattr(L, f).argtypes = [ctypes.c_double, ctypes.c_double]
                getattr(L, f).restype = ctypes.c_double
            _lib = L
    return _lib


def as_const(k) -> OracleStepConst:
    """Copy any 216-byte StepConst-layout structure into the oracle's type."""
    assert ctypes.sizeof(k) == ctypes.sizeof(OracleStepConst) == 216
    return OracleStepConst.from_buffer_copy(bytes(k))


def step(T: np.ndarray, k, phys: int = 0, bc: int = 0, T_D: float = 300.0) -> np.ndarray:
    T = np.ascontiguousarray(T, dtype=np.float64)
    out = np.empty_like(T)
    kk = as_const(k)
    lib().oracle_step(_ptr(T), _ptr(out), ctypes.byref(kk), phys, bc, T_D)
    return out


def reduce(T: np.ndarray, nx: int, ny: int, Tm: float):
    T = np.ascontiguousarray(T, dtype=np.float64)
    p = OraclePartial()
    lib().oracle_reduce(_ptr(T), nx, ny, Tm, ctypes.byref(p))
    return (p.tmax, p.arg, p.ymin, p.ymax)


def measure(T: np.ndarray, nx: int, ny: int, dy: float, Tm: float):
    T = np.ascontiguousarray(T, dtype=np.float64)
    m = OracleMeasure()
    lib().oracle_measure(_ptr(T), nx, ny, dy, Tm, ctypes.byref(m))
    return dict(peak_T=m.peak_T, x_hot=m.x_hot, W_um=m.W_um, W_sub_um=m.W_sub_um)


def w_sub(col: np.ndarray, dy: float, Tm: float) -> float:
    col = np.ascontiguousarray(col, dtype=np.float64)
    return lib().oracle_w_sub(_ptr(col), len(col), dy, Tm)


def run(T0: np.ndarray, k, laser: np.ndarray, phys: int = 0, bc: int = 0,
        T_D: float = 300.0, Tm: float = 1609.0, with_ring: bool = True):
    """Advance T0 by len(laser) steps; laser is (n, 3) (x_l, y_l, q_scale).
    Returns (final field, per-step partials as a PARTIAL_DTYPE array)."""
    a = np.array(T0, dtype=np.float64, copy=True, order="C")
    b = np.empty_like(a)
    laser = np.ascontiguousarray(laser, dtype=np.float64)
    n = laser.shape[0]
    ring = np.zeros(n, dtype=PARTIAL_DTYPE) if with_ring else None
    kk = as_const(k)
    which = lib().oracle_run(_ptr(a), _ptr(b), ctypes.byref(kk), _ptr(laser), n, phys, bc,
                             T_D, Tm, ring.ctypes.data if ring is not None else None)
    return (b if which else a), ring


def run_quiet(T0: np.ndarray, k, laser: np.ndarray, bc: int = 0, T_D: float = 300.0,
              Tm: float = 1609.0, with_ring: bool = True, threads: int | None = None,
              probe: np.ndarray | None = None):
    """``run`` for the baseline physics, computing per step only the cells
    that can differ from the quiet temperature Tamb (= Tsub) and sharing
    them among threads: bit-identical results, far less work on large
    fields heated along a track.  Raises when its preconditions (Tamb ==
    Tsub, fixed edges at Tamb, Tm >= Tamb) do not hold.

    probe (optional, one flat index per step): also returns the field's
    value at probe[s] after step s, as a third result."""
    a = np.array(T0, dtype=np.float64, copy=True, order="C")
    b = np.empty_like(a)
    laser = np.ascontiguousarray(laser, dtype=np.float64)
    n = laser.shape[0]
    ring = np.zeros(n, dtype=PARTIAL_DTYPE) if with_ring else None
    kk = as_const(k)
    nt = threads or min(64, os.cpu_count() or 1)
    pidx = pval = None
    if probe is not None:
        pidx = np.ascontiguousarray(probe, dtype=np.int64)
        assert pidx.shape == (n,)
        pval = np.full(n, np.nan)
    which = lib().oracle_run_quiet(_ptr(a), _ptr(b), ctypes.byref(kk), _ptr(laser), n, bc, T_D,
                                   Tm, ring.ctypes.data if ring is not None else None, nt,
                                   pidx.ctypes.data if pidx is not None else None,
                                   pval.ctypes.data if pval is not None else None)
    if which < 0:
        raise ValueError("run_quiet needs Tamb == Tsub, fixed edges at Tamb and Tm >= Tamb")
    T = b if which else a
    return (T, ring, pval) if probe is not None else (T, ring)


# ---- the reference's own code (oracle/_ref) --------------------------------

def reference_tree() -> str | None:
    """The reference source tree: $LPBF_REFERENCE, else the location the last
    ``make -C oracle ref`` run by the build recorded in oracle/_ref, else
    None (no default path)."""
    env = os.environ.get("LPBF_REFERENCE")
    if env:
        return env
    rec = os.path.join(_REF, "REFERENCE_TREE")
    if os.path.exists(rec):
        with open(rec) as f:
            p = f.read().strip()
        return p or None
    return None


def have_reference() -> bool:
    return all(os.path.exists(os.path.join(_REF, f))
               for f in ("libref.so", "libref_hh.so", "libref_plan.so"))


def ref_lib(name: str = "libref.so"):
    with _lock:
        if name not in _ref:
            path = os.path.join(_REF, name)
            if not os.path.exists(path):
                raise FileNotFoundError(f"{path} is not built (make -C oracle ref)")
            L = ctypes.CDLL(path)
            if name == "libref.so":
                sc = ctypes.POINTER(OracleStepConst)
                L.ref_cpu_step.argtypes = [_dp, _dp, sc, ctypes.c_int]
                L.ref_cpu_run_plan.argtypes = [_dp, sc, _dp, ctypes.c_int, ctypes.c_int]
                L.ref_measure_host.argtypes = [_dp, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                               ctypes.c_double, ctypes.c_double, _dp, _dp, _dp,
                                               ctypes.POINTER(ctypes.c_int)]
                L.ref_run_cpu.argtypes = [_dp, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                          ctypes.c_double, _dp, _dp, ctypes.c_int,
                                          ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_double, _dp, _dp, _dp]
                L.ref_run_cpu.restype = ctypes.c_double
                L.ref_make_const.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                             ctypes.c_double, _dp, _dp, ctypes.c_int,
                                             ctypes.c_double, sc]
                L.ref_dt_cfl.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                         ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_double, ctypes.c_int, ctypes.c_double]
                L.ref_dt_cfl.restype = ctypes.c_double
            elif name == "libref_hh.so":
                L.ref_hh_run.argtypes = [_dp, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                         ctypes.c_double, _dp, _dp, ctypes.c_int,
                                         ctypes.c_double, _dp, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                         ctypes.c_double, ctypes.c_void_p]
                L.ref_hh_run.restype = ctypes.c_double
            elif name == "libref_plan.so":
                L.ref_build_plan.argtypes = [ctypes.c_double] * 5 + [ctypes.c_int, ctypes.c_int,
                                             ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_void_p]
                L.ref_build_plan.restype = ctypes.c_int
                L.ref_gpu_task_run.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                               ctypes.c_double, ctypes.POINTER(OracleStepConst),
                                               ctypes.c_double, ctypes.c_double,
                                               ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                               ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp]
                L.ref_gpu_task_run.restype = ctypes.c_double
            _ref[name] = L
    return _ref[name]


def mat6(mat) -> np.ndarray:
    return np.array([mat.k, mat.rho, mat.cp, mat.Tm, mat.eps, mat.eta], dtype=np.float64)


def pr8(pr) -> np.ndarray:
    return np.array([pr.P, pr.V, pr.r0, pr.h, pr.hConv, pr.dSub, pr.Tamb, pr.Tsub],
                    dtype=np.float64)


def ref_step(T: np.ndarray, k, phys: int = 0) -> np.ndarray:
    T = np.ascontiguousarray(T, dtype=np.float64)
    out = np.empty_like(T)
    kk = as_const(k)
    ref_lib().ref_cpu_step(_ptr(T), _ptr(out), ctypes.byref(kk), phys)
    return out


def ref_run_plan(T0: np.ndarray, k, laser: np.ndarray, phys: int = 0) -> np.ndarray:
    T = np.array(T0, dtype=np.float64, copy=True, order="C")
    laser = np.ascontiguousarray(laser, dtype=np.float64)
    kk = as_const(k)
    ref_lib().ref_cpu_run_plan(_ptr(T), ctypes.byref(kk), _ptr(laser), laser.shape[0], phys)
    return T


def ref_make_const(mat, pr, dom, dt) -> OracleStepConst:
    out = OracleStepConst()
    m, p = mat6(mat), pr8(pr)
    ref_lib().ref_make_const(dom.nx, dom.ny, dom.Lx, dom.Ly, _ptr(m), _ptr(p),
                             int(pr.radiation), dt, ctypes.byref(out))
    return out


def ref_dt_cfl(mat, dom, ext: bool = False, kmult: float = 1.0) -> float:
    return ref_lib().ref_dt_cfl(dom.nx, dom.ny, dom.Lx, dom.Ly, mat.k, mat.rho, mat.cp,
                                int(ext), kmult)


def ref_run_cpu(mat, pr, dom, dt, n_steps, phys=0, kmult=1.0):
    """The reference run_cpu() (its built-in single-track law)."""
    T = np.empty(dom.nx * dom.ny, dtype=np.float64)
    pk, pw, ws = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    m, p = mat6(mat), pr8(pr)
    wall = ref_lib().ref_run_cpu(_ptr(T), dom.nx, dom.ny, dom.Lx, dom.Ly, _ptr(m), _ptr(p),
                                 int(pr.radiation), dt, n_steps, phys, kmult,
                                 ctypes.byref(pk), ctypes.byref(pw), ctypes.byref(ws))
    return dict(T=T.reshape(dom.ny, dom.nx), peak_T=pk.value, peak_W=pw.value,
                steady_W_sub=ws.value, wall_ms=wall)


def ref_gpu_task_run(k, dom, plan: np.ndarray, Tm: float, Tamb: float, batch: int = 64,
                     mode: int = 2, fused: bool = False, pinned: bool = False):
    """The reference's own GpuStepTask graph (its kernels, built for sm_100a)
    over ``plan`` (Tick array) on the current CUDA device.  Returns (wall ms
    from the first Tick to the graph's end, the run's peak temperature)."""
    plan = np.ascontiguousarray(plan)
    assert plan.dtype.itemsize == 56
    kk = as_const(k)
    pk = ctypes.c_double()
    ms = ref_lib("libref_plan.so").ref_gpu_task_run(
        dom.nx, dom.ny, dom.Lx, dom.Ly, ctypes.byref(kk), Tm, Tamb, plan.ctypes.data,
        len(plan), batch, mode, int(fused), int(pinned), ctypes.byref(pk))
    return ms, pk.value


def ref_build_plan(pr, dom, dt, n_steps, snap_every, tick_dtype) -> np.ndarray:
    out = np.zeros(n_steps, dtype=tick_dtype)
    ref_lib("libref_plan.so").ref_build_plan(pr.P, pr.V, pr.r0, dom.Lx, dom.Ly, dom.nx,
                                             dom.ny, dt, n_steps, snap_every,
                                             out.ctypes.data)
    return out


def ref_hh_run(T0: np.ndarray, mat, pr, dom, dt, laser: np.ndarray, n_threads: int,
               n_tiles: int, phys: int = 0, kmult: float = 1.0, Tm: float = 1609.0,
               want_trace: bool = False):
    """The reference StepTileTask over n_tiles row strips on n_threads workers.
    Returns (final field, wall seconds, peak trace or None)."""
    T = np.array(T0, dtype=np.float64, copy=True, order="C")
    laser = np.ascontiguousarray(laser, dtype=np.float64)
    trace = np.zeros(laser.shape[0]) if want_trace else None
    m, p = mat6(mat), pr8(pr)
    wall = ref_lib("libref_hh.so").ref_hh_run(
        _ptr(T), dom.nx, dom.ny, dom.Lx, dom.Ly, _ptr(m), _ptr(p), int(pr.radiation), dt,
        _ptr(laser), laser.shape[0], n_threads, n_tiles, phys, kmult, Tm,
        trace.ctypes.data if trace is not None else None)
    return T, wall, trace
