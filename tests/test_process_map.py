# SPDX-License-Identifier: 0BSD
"""Process-map scenario draws and the batch's host-side layout (no GPU)."""
import ctypes
import math
import subprocess

import numpy as np
import pytest

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
    scs = PM.process_map(6, 20)
    arr = (_lib.Scenario * len(scs))()
    plans = [np.ascontiguousarray(s.plan) for s in scs]
    for i, s in enumerate(scs):
        arr[i].k = ctypes.pointer(s.k)
        arr[i].plan = plans[i].ctypes.data
    b1 = L.lpbf_b200_batch_workspace_bytes(arr, len(scs), 10, ctypes.byref(batch_opts(depth=3)))
    b2 = L.lpbf_b200_batch_workspace_bytes(arr, len(scs), 20, ctypes.byref(batch_opts(depth=3)))
    assert b1 > 0 and b1 % 256 == 0
    assert b2 - b1 >= 10 * len(scs) * 40 - 256    # 40-byte per-step laser records
    small = L.lpbf_b200_batch_workspace_bytes(arr, len(scs), 10,
                                              ctypes.byref(batch_opts(rows=(96, 96, 96, 96))))
    assert small < b1                             # fewer tasks, fewer partials
    # without the plans the size is a bound that holds for any plan
    for i in range(len(scs)):
        arr[i].plan = None
    assert L.lpbf_b200_batch_workspace_bytes(arr, len(scs), 10,
                                             ctypes.byref(batch_opts(depth=3))) >= b1
    assert L.lpbf_b200_batch_workspace_bytes(arr, len(scs), 10,
                                             ctypes.byref(batch_opts(depth=9))) == 0


def test_tune_cache_round_trip(tmp_path):
    from hedgehog_lpbf_b200.batch import batch_opts, opts_dict
    L = _lib.lib()
    path = str(tmp_path / "tune.json").encode()
    out = _lib.BatchOpts()
    assert L.lpbf_b200_tune_cache_get(path, b"gpu|sm148|classes 64,64,64,64", ctypes.byref(out)) == 1
    o1 = batch_opts(depth=2, ctas_per_sm=2, rows=(24, 48, 96, 192), staging=1)
    o2 = batch_opts(depth=3, rows=(12, 12, 24, 24), staging=2)
    assert L.lpbf_b200_tune_cache_put(path, b"k1", ctypes.byref(o1), 241.5) == 0
    assert L.lpbf_b200_tune_cache_put(path, b'k "2"', ctypes.byref(o2), 300.0) == 0
    assert L.lpbf_b200_tune_cache_get(path, b"k1", ctypes.byref(out)) == 0
    assert opts_dict(out) == opts_dict(o1)
    assert L.lpbf_b200_tune_cache_get(path, b'k "2"', ctypes.byref(out)) == 0
    assert opts_dict(out) == opts_dict(o2)
    import json
    doc = json.load(open(path.decode()))          # the file is plain JSON
    assert doc["version"] == 1 and doc["entries"]["k1"]["rows"] == [24, 48, 96, 192]
    assert doc["entries"]["k1"]["gcells"] == 241.5
    # replacing a key keeps the others
    assert L.lpbf_b200_tune_cache_put(path, b"k1", ctypes.byref(o2), 1.0) == 0
    assert L.lpbf_b200_tune_cache_get(path, b"k1", ctypes.byref(out)) == 0
    assert opts_dict(out) == opts_dict(o2)
    assert L.lpbf_b200_tune_cache_get(path, b'k "2"', ctypes.byref(out)) == 0
    # a malformed file is an error for get and is rewritten by put
    open(path.decode(), "w").write("{not json")
    assert L.lpbf_b200_tune_cache_get(path, b"k1", ctypes.byref(out)) == -1
    assert L.lpbf_b200_tune_cache_put(path, b"k3", ctypes.byref(o1), 2.0) == 0
    assert L.lpbf_b200_tune_cache_get(path, b"k3", ctypes.byref(out)) == 0


def test_tune_key_is_the_size_class_histogram():
    from hedgehog_lpbf_b200.batch import tune_key
    scs = PM.process_map(40, 2)
    key = tune_key(scs)
    counts = [0, 0, 0, 0]
    for s in scs:
        counts[_lib.lib().lpbf_b200_batch_size_class(s.k.nx, s.k.ny)] += 1
    pow2 = [0 if c == 0 else 1 << (c - 1).bit_length() for c in counts]
    assert key.endswith("classes " + ",".join(map(str, pow2)))


def test_summarize_melt_results():
    from hedgehog_lpbf_b200.solver import PARTIAL_DTYPE
    r = np.zeros(5, dtype=PARTIAL_DTYPE)
    r["tmax"] = [400.0, 1800.0, 2100.0, 1650.0, 1200.0]
    r["ymin"] = [90, 40, 38, 45, 90]
    r["ymax"] = [-1, 44, 47, 46, -1]
    s = PM.summarize(r, 5e-6)
    assert s["peak_T_K"] == 2100.0 and s["peak_step"] == 2
    assert s["first_melt_step"] == 1 and s["molten_steps"] == 3
    assert s["max_melt_rows"] == 10 and abs(s["max_melt_extent_um"] - 50.0) < 1e-9
    none = np.zeros(2, dtype=PARTIAL_DTYPE)
    none["ymax"] = -1
    assert PM.summarize(none, 5e-6)["first_melt_step"] == -1


def test_process_map_cli_rejects_bad_arguments():
    with pytest.raises(SystemExit):
        PM.main(["--scenarios", "0"])
    with pytest.raises(SystemExit):
        PM.main(["--rows", "1,2", "--depth", "2", "--steps", "0"])


@pytest.mark.gpu
def test_process_map_cli_runs_and_writes_csv(gpu, tmp_path):
    out = tmp_path / "pm.csv"
    rc = PM.main(["--scenarios", "2", "--steps", "6", "--side", "256", "--depth", "2",
                  "--rows", "12,12,12,12", "--out", str(out)])
    assert rc == 0
    lines = out.read_text().strip().splitlines()
    assert lines[0].split(",") == list(PM.COLUMNS)
    assert len(lines) == 3
    for line in lines[1:]:
        row = dict(zip(PM.COLUMNS, line.split(",")))
        assert int(row["side"]) == 256 and int(row["steps"]) == 6
        assert float(row["peak_T_K"]) > 300.0
