# SPDX-License-Identifier: 0BSD
"""Generate the golden fixtures in tests/golden/ from the reference itself.

Run in a checkout where the reference tree is available (LPBF_REFERENCE, or
the location recorded by ``make -C oracle ref`` through the build) after
building oracle/_ref:

    python tests/golden/make_golden.py

Writes
  case0.json       the reference's committed case-0 outputs
                   (reference/case0/metrics.csv, reference/case0/meta.json)
  ref_small.npz    final fields of the reference's own cpu_step
                   (src/gpu/lpbf_cuda.cu:154-210, compiled from the reference
                   tree into oracle/_ref/libref.so) on small grids, its
                   measure_host() results, its make_const() bytes and its
                   build_plan() Ticks.
"""
from __future__ import annotations

import csv
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from hedgehog_lpbf_b200 import params as P  # noqa: E402
from hedgehog_lpbf_b200 import plan as PL  # noqa: E402
from oracle import oracle as O  # noqa: E402

REF = O.reference_tree()
if not REF:
    sys.exit("make_golden.py: set LPBF_REFERENCE to the reference source tree")


def case0():
    rows = []
    with open(os.path.join(REF, "reference/case0/metrics.csv")) as f:
        for r in csv.DictReader(f):
            rows.append({k: float(v) for k, v in r.items()})
    with open(os.path.join(REF, "reference/case0/meta.json")) as f:
        meta = json.load(f)
    return {"metrics": rows, "meta": meta}


# Small cases: (name, nx, ny, Lx, Ly, n_steps, phys, laser placement, q pattern)
CASES = [
    ("mirror_64x48", 64, 48, 63 * 5e-6, 47 * 5e-6, 40, 0, "centre", "on"),
    ("mirror_odd_33x17", 33, 17, 32 * 5e-6, 16 * 5e-6, 25, 0, "corner", "on"),
    ("mirror_130x70_edge", 130, 70, 129 * 5e-6, 69 * 5e-6, 30, 0, "edge", "pulsed"),
    ("ext_48x40", 48, 40, 47 * 5e-6, 39 * 5e-6, 30, 1, "centre", "on"),
    ("ext_kmult_40x24", 40, 24, 39 * 5e-6, 23 * 5e-6, 20, 1, "moving", "on"),
]


def laser_for(kind, dom, n, qpat):
    las = np.zeros((n, 3))
    for s in range(n):
        if kind == "centre":
            x, y = 0.5 * dom.Lx, 0.5 * dom.Ly
        elif kind == "corner":
            x, y = 0.0, 0.0
        elif kind == "edge":
            x, y = dom.Lx, 0.3 * dom.Ly
        else:
            x, y = (0.1 + 0.8 * s / max(1, n - 1)) * dom.Lx, 0.45 * dom.Ly
        q = 1.0 if qpat == "on" else (1.0 if (s // 3) % 2 == 0 else 0.0)
        las[s] = (x, y, q)
    return las


def small_cases(out):
    mat = P.Material(k=20.0, rho=7900.0, cp=500.0, Tm=1609.0, eta=0.4)
    pr = P.Process(P=200.0, V=1.0, r0=50e-6, h=50e-6, Tamb=300.0, Tsub=300.0)
    for name, nx, ny, Lx, Ly, n, phys, kind, qpat in CASES:
        dom = P.Domain(Lx=Lx, Ly=Ly, nx=nx, ny=ny)
        dt = P.dt_cfl(mat, dom) if phys == 0 else O.ref_dt_cfl(mat, dom, ext=True,
                                                                 kmult=2.0 if "kmult" in name else 1.0)
        k = O.ref_make_const(mat, pr, dom, dt)
        if "kmult" in name:
            k.kmult = 2.0
        las = laser_for(kind, dom, n, qpat)
        T0 = np.full(nx * ny, pr.Tamb)
        # a non-uniform start so that every term of the update is exercised
        rng = np.random.default_rng(7)
        T0 += rng.uniform(0.0, 900.0, size=T0.shape)
        T = O.ref_run_plan(T0, k, las, phys=phys)
        pk, wu, ws, xh = (np.zeros(1), np.zeros(1), np.zeros(1), np.zeros(1, dtype=np.int32))
        import ctypes
        L = O.ref_lib()
        a, b, c = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        d = ctypes.c_int()
        L.ref_measure_host(T.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), nx, ny, Lx, Ly,
                           1609.0, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c), ctypes.byref(d))
        out[f"{name}/T0"] = T0
        out[f"{name}/laser"] = las
        out[f"{name}/const"] = np.frombuffer(bytes(k), dtype=np.uint8)
        out[f"{name}/phys"] = np.array(phys)
        out[f"{name}/T"] = T
        out[f"{name}/measure"] = np.array([a.value, b.value, c.value, d.value])


def consts_and_plans(out):
    # make_const bytes for the case table and the benchmark constants
    for cid in P.CASES:
        mat, dom = P.Material(), P.Domain()
        pr = P.apply_case(cid, P.Process())
        dt = O.ref_dt_cfl(mat, dom)
        out[f"const_case{cid}"] = np.frombuffer(bytes(O.ref_make_const(mat, pr, dom, dt)), np.uint8)
        out[f"dt_case{cid}"] = np.array(dt)
    mat, pr = P.benchmark_material_process()
    for n in (512, 8192):
        dom = P.square_domain(n)
        dt = P.dt_fraction(mat, dom)
        out[f"const_bench{n}"] = np.frombuffer(bytes(O.ref_make_const(mat, pr, dom, dt)), np.uint8)
    # reference build_plan for case 0 (1427 steps, snap every 200)
    mat, dom = P.Material(), P.Domain()
    pr = P.apply_case("0", P.Process())
    dt = O.ref_dt_cfl(mat, dom)
    n = int(1.5e-3 / dt)
    out["plan_case0"] = O.ref_build_plan(pr, dom, dt, n, 200, PL.TICK_DTYPE).view(np.uint8)
    out["dt_ext_kmult2"] = np.array(O.ref_dt_cfl(mat, dom, ext=True, kmult=2.0))


def main():
    if not O.have_reference():
        sys.exit("oracle/_ref is not built: run `make -C oracle ref` with the reference tree")
    with open(os.path.join(HERE, "case0.json"), "w") as f:
        json.dump(case0(), f, indent=1)
    out = {}
    small_cases(out)
    consts_and_plans(out)
    np.savez_compressed(os.path.join(HERE, "ref_small.npz"), **out)
    print("wrote", sorted(out)[:5], "...", len(out), "arrays")


if __name__ == "__main__":
    main()
