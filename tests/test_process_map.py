# SPDX-License-Identifier: 0BSD
"""Process-map scenario draws and the batch's host-side layout (no GPU)."""
import ctypes
import math
import subprocess

import numpy as np

from hedgehog_lpbf_b200 import _lib
from hedgehog_lpbf_b200 import process_map as PM


def test_mt19937_64_known_answer():
    # The C++ standard fixes the 10000th output of a default-seeded
    # std::mt19937_64 (seed 5489) at 9981545732273789042.
    g = PM.MT19937_64(5489)
    for _ in range(9999):
        g()
    assert g() == 9981545732273789042


def test_draws_match_std_mt19937_64(tmp_path):
    """The same draws from a C++ program on std::mt19937_64."""
    src = tmp_path / "d.cpp"
    src.write_text(
        "#include <random>\n#include <cstdio>\n#include <cstdint>\n"
        "static double u(uint64_t x){ return (double)(x >> 11) * (1.0 / 9007199254740992.0); }\n"
        "int main(){ const int sides[4] = {256, 512, 1024, 2048};\n"
        " for (int i = 0; i < 40; ++i) { std::mt19937_64 g((uint64_t)i);\n"
        "  int side = sides[g() >> 62]; double P = 100.0 + 300.0 * u(g());\n"
        "  double V = 0.5 + 1.5 * u(g()); double r0 = 35e-6 + 35e-6 * u(g());\n"
        "  double a = 3.141592653589793 * u(g()); double h = 80e-6 + 40e-6 * u(g());\n"
        "  std::printf(\"%d %a %a %a %a %a\\n\", side, P, V, r0, a, h); } }\n")
    exe = tmp_path / "d"
    subprocess.run(["g++", "-O2", "-std=c++17", str(src), "-o", str(exe)], check=True)
    lines = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    for i in range(40):
        d = PM.draw(i)
        f = lines[i].split()
        assert int(f[0]) == d.side
        assert [float.fromhex(x) for x in f[1:]] == [d.P, d.V, d.r0, d.angle, d.hatch]


def test_draw_ranges_and_size_mix():
    ds = [PM.draw(i) for i in range(256)]
    assert all(100 <= d.P < 400 and 0.5 <= d.V < 2 and 35e-6 <= d.r0 < 70e-6 for d in ds)
    assert all(0 <= d.angle < math.pi and 80e-6 <= d.hatch < 120e-6 for d in ds)
    counts = {s: sum(d.side == s for d in ds) for s in PM.SIDES}
    assert all(40 <= c <= 90 for c in counts.values()), counts
    assert PM.cells(256) == sum(d.side ** 2 for d in ds)


def test_raster_stays_inside_the_domain():
    for i in range(16):
        d = PM.draw(i)
        k, plan, _ = PM.scenario_inputs(d, 4000, side=256)
        L = (k.nx - 1) * k.dx
        assert (plan["q_scale"] > 0).any()
        assert np.all(plan["x_l"] > 0.05 * L) and np.all(plan["x_l"] < 0.95 * L)
        assert np.all(plan["y_l"] > 0.05 * L) and np.all(plan["y_l"] < 0.95 * L)


def test_batch_size_classes_and_workspace_bytes():
    from hedgehog_lpbf_b200.batch import batch_opts
    L = _lib.lib()
    assert [L.lpbf_b200_batch_size_class(s, s) for s in (256, 511, 512, 1024, 2047, 2048, 8192)] \
        == [0, 0, 1, 2, 2, 3, 3]
    assert L.lpbf_b200_batch_size_class(100, 3000) == 3
    scs = PM.process_map(6, 10)
    arr = (_lib.Scenario * len(scs))()
    for i, s in enumerate(scs):
        arr[i].k = ctypes.pointer(s.k)
    b1 = L.lpbf_b200_batch_workspace_bytes(arr, len(scs), 10, ctypes.byref(batch_opts(depth=3)))
    b2 = L.lpbf_b200_batch_workspace_bytes(arr, len(scs), 20, ctypes.byref(batch_opts(depth=3)))
    assert b1 > 0 and b1 % 256 == 0
    assert b2 - b1 >= 10 * len(scs) * 40 - 256    # 40-byte per-step laser records
    small = L.lpbf_b200_batch_workspace_bytes(arr, len(scs), 10,
                                              ctypes.byref(batch_opts(rows=(96, 96, 96, 96))))
    assert small < b1                             # fewer tasks, fewer partials
    assert L.lpbf_b200_batch_workspace_bytes(arr, len(scs), 10,
                                             ctypes.byref(batch_opts(depth=9))) == 0
