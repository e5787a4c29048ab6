"""The parts of bench.py's JSON line that are computed on the host, checked
on CPU: the clock summary (a throttled or clock-locked run must show in the
line), the roofline of the bulge-chasing launch (algorithmic bytes from the
task count of every sweep), and the whole-step FP64 work of the reference's
method."""
import os
import sys
from types import SimpleNamespace

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def test_clock_summary_reports_median_and_reasons():
    import bench
    clk = bench.ClockSampler(0)
    clk.lines = [
        "0, 1965, 1965, 820.5, 0x0, Not Active, Not Active, Not Active, Not Active",
        "0, 1950, 1965, 990.1, 0x4, Not Active, Not Active, Not Active, Active",
        "0, 1965, 1965, 700.0, 0x0, Not Active, Not Active, Not Active, Not Active",
        "garbage line",
    ]
    s = clk.summary()
    assert s["samples"] == 3
    assert s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"]
    clk.lines = ["0, 1200, 1965, 500.0, 0x8, Active, Not Active, Active, Not Active"]
    assert clk.summary()["reasons"] == ["hw_slowdown", "sw_thermal_slowdown"]


def test_chase_roofline_counts_every_task():
    import bench
    sizes = [10, 20]                         # atoms; bands of n = 30 and 60
    stage = {"total": 5.0, "setup": 0.01, "relay_build": 0.1, "relay_solve": 1.0, "tridiag": 3.0,
             "eig_energy": 0.2, "tridiag_dense_to_band": 1.0, "tridiag_to_tridiagonal": 2.0,
             "tridiag_one_stage_launch": 0.0, "tridiag_band_chase_launch": 2.0}
    r = bench.roofline(stage, sizes, "mixed_learned")
    tasks = 0
    for N in sizes:                          # brute force: one task per 32 rows below each sweep's column
        n = 3 * N
        for i in range(n - 2):
            rows = n - i - 1
            tasks += -(-rows // 32)
    nbytes = tasks * 2 * 2 * 32 * 32 * 8
    assert r["kernel_ms"] == 2.0
    assert r["achieved"] == pytest.approx(nbytes / 2e-3 / 1e9)
    assert r["frac"] == pytest.approx(r["achieved"] / r["peak"])
    for key in ("bound", "unit", "traffic", "peak_source", "algorithmic"):
        assert key in r


def test_step_flops_follow_the_reference_method():
    import bench
    res = [SimpleNamespace(alpha_eff=np.zeros(100), supercell=(1, 1, 1)),
           SimpleNamespace(alpha_eff=np.zeros(20), supercell=(2, 2, 1))]
    expect = 0.0
    for N, nsl in ((100, 1), (20, 4)):
        n = 3.0 * N
        expect += 21 * n ** 3 / 3 + 126 * n * n + 4.0 / 3.0 * (n * nsl) ** 3
    assert bench.fp64_step_flops(res) == pytest.approx(expect)
