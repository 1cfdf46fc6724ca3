# SPDX-License-Identifier: 0BSD
"""Host-side mirror of the reference's parameter and ABI types.

``Material``/``Process``/``Domain`` and ``dt_cfl`` follow the reference's
include/params.hpp:13-47 (same fields, defaults and arithmetic);
``StepConst``/``Partial`` are ctypes structures with the exact byte layout of
include/lpbf_step_const.hpp:19-33 (216 and 24 bytes) and ``make_const``
follows lpbf_step_const.hpp:36-54 operation by operation, so the doubles it
produces are bit-identical to the reference's.  ``Tick`` mirrors
include/gpu_messages.hpp:18-26 (56 bytes).
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, replace

SIGMA_SB = 5.670374419e-8


@dataclass
class Material:
    k: float = 25.0
    rho: float = 8190.0
    cp: float = 565.0
    Tm: float = 1609.0
    eps: float = 0.40
    eta: float = 0.35

    def alpha(self) -> float:
        return self.k / (self.rho * self.cp)


@dataclass
class Process:
    P: float = 285.0
    V: float = 0.96
    r0: float = 33.5e-6
    h: float = 40.0e-6
    hConv: float = 100.0
    dSub: float = 30.0e-6
    Tamb: float = 298.15
    Tsub: float = 298.15
    radiation: bool = True


@dataclass
class Domain:
    Lx: float = 1.6e-3
    Ly: float = 0.6e-3
    nx: int = 240
    ny: int = 120

    def dx(self) -> float:
        return self.Lx / (self.nx - 1)

    def dy(self) -> float:
        return self.Ly / (self.ny - 1)


def dt_cfl(mat: Material, dom: Domain) -> float:
    """params.hpp:44-47: 0.35 of the 2D explicit diffusion limit."""
    sx = 1.0 / (dom.dx() * dom.dx())
    sy = 1.0 / (dom.dy() * dom.dy())
    return 0.35 / (mat.alpha() * (sx + sy))


class StepConst(ctypes.Structure):
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
        ("radiation", ctypes.c_bool),
        ("kmult", ctypes.c_double),
        ("x_l", ctypes.c_double), ("y_l", ctypes.c_double),
        ("q_scale", ctypes.c_double),
    ]


class Partial(ctypes.Structure):
    _fields_ = [("tmax", ctypes.c_double), ("arg", ctypes.c_longlong),
                ("ymin", ctypes.c_int), ("ymax", ctypes.c_int)]


class Tick(ctypes.Structure):
    _fields_ = [("step", ctypes.c_int), ("t", ctypes.c_double),
                ("x_l", ctypes.c_double), ("y_l", ctypes.c_double),
                ("q_scale", ctypes.c_double), ("x_laser_csv", ctypes.c_double),
                ("wrapped", ctypes.c_bool), ("dump", ctypes.c_bool)]


assert ctypes.sizeof(StepConst) == 216 and StepConst.radiation.offset == 176
assert ctypes.sizeof(Partial) == 24
assert ctypes.sizeof(Tick) == 56 and Tick.wrapped.offset == 48


def make_const(mat: Material, pr: Process, dom: Domain, dt: float) -> StepConst:
    """lpbf_step_const.hpp:36-54 (same operations in the same order)."""
    k = StepConst()
    k.nx, k.ny = dom.nx, dom.ny
    k.dx, k.dy = dom.dx(), dom.dy()
    k.inv_dx2 = 1.0 / (k.dx * k.dx)
    k.inv_dy2 = 1.0 / (k.dy * k.dy)
    k.inv_r0_sq = 1.0 / (pr.r0 * pr.r0)
    k.alpha = mat.alpha()
    k.K, k.rho, k.cp = mat.k, mat.rho, mat.cp
    k.rho_cp = mat.rho * mat.cp
    k.inv_h = 1.0 / pr.h
    k.h = pr.h
    k.dt = dt
    k.peak_S = (2.0 * mat.eta * pr.P) / (math.pi * pr.r0 * pr.r0)
    k.eta, k.P = mat.eta, pr.P
    k.hConv, k.Tamb, k.Tsub, k.dSub = pr.hConv, pr.Tamb, pr.Tsub, pr.dSub
    k.eps = mat.eps
    k.radiation = bool(pr.radiation)
    k.kmult = 1.0
    k.q_scale = 1.0
    k.x_l = 0.0
    k.y_l = 0.0
    return k


# AMB2022-03 IN718 single-track cases (src/main.cpp:97-109).
CASES = {
    "0":   dict(P=285.0, V=0.96, r0=33.5e-6),
    "1.1": dict(P=285.0, V=0.96, r0=24.5e-6),
    "1.2": dict(P=285.0, V=0.96, r0=41.0e-6),
    "2.1": dict(P=285.0, V=1.20, r0=33.5e-6),
    "2.2": dict(P=285.0, V=0.80, r0=33.5e-6),
    "3.1": dict(P=325.0, V=0.96, r0=33.5e-6),
    "3.2": dict(P=245.0, V=0.96, r0=33.5e-6),
}


def apply_case(case_id: str, pr: Process) -> Process:
    if case_id not in CASES:
        raise ValueError(f"unknown case '{case_id}'")
    return replace(pr, **CASES[case_id])


def benchmark_material_process(P=200.0, V=1.0, r0=50e-6):
    """The constants of the 512^2 / 8192^2 / 4096^2 workloads: k=20 W/m/K,
    rho=7900, cp=500, 50 um layer, absorptivity 0.4, T0 = Tamb = Tsub = 300 K,
    reference loss terms (convection 100 W/m^2/K, emissivity 0.4, substrate
    at 30 um) and a 1700 K melt threshold."""
    mat = Material(k=20.0, rho=7900.0, cp=500.0, Tm=1700.0, eps=0.40, eta=0.4)
    pr = Process(P=P, V=V, r0=r0, h=50e-6, hConv=100.0, dSub=30e-6,
                 Tamb=300.0, Tsub=300.0, radiation=True)
    return mat, pr


def square_domain(n: int, dx: float = 5e-6) -> Domain:
    """n x n nodes at spacing dx (Lx = (n-1) dx, the reference's node law)."""
    return Domain(Lx=(n - 1) * dx, Ly=(n - 1) * dx, nx=n, ny=n)


def dt_fraction(mat: Material, dom: Domain, frac: float = 0.2) -> float:
    """dt = frac * dx^2 / alpha (the benchmark workloads use frac = 0.2)."""
    return frac * dom.dx() * dom.dx() / mat.alpha()
