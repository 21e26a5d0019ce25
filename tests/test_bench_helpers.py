"""The measurement arithmetic of bench.py on the CPU: the non-walk stages' HBM
roofline (algorithmic bytes per particle, cell and group; the reference's
IOCOUNT build accounting) and the log-log interpolation of the fixed-angle
sweep at equal error that the learned form is judged against."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def test_hbm_roofline_bytes_and_fraction():
    import bench
    n, info, ms = 1 << 20, {"ncells": 250000, "ngroups": 17000, "nlevels": 12}, 0.5
    r = bench.hbm_roofline(n, info, ms)
    want = n * (28 + 24 + 64 + 8 + 16 + 8 + 80) + 250000 * (16 + 72) + 8 * 17000
    assert r["algorithmic_bytes_per_step"] == want
    assert r["achieved"] == pytest.approx(want / (ms * 1e-3) / 1e9)
    assert r["frac"] == pytest.approx(r["achieved"] / r["peak"])
    assert r["reference_build_bytes"] == 32.0 * n * 12
    assert r["bound"] == "hbm" and r["unit"] == "GB/s"


def test_at_equal_interpolates_log_log_inside_the_sweep_only():
    import bench
    sweep = [{"v": 100.0, "e": 1e-4}, {"v": 400.0, "e": 1e-3}, {"v": 200.0, "e": 3e-4}]
    # exact at the points, log-log linear between them
    assert bench.at_equal(sweep, "v", "e", 1e-4) == pytest.approx(100.0)
    assert bench.at_equal(sweep, "v", "e", 1e-3) == pytest.approx(400.0)
    mid = np.sqrt(3e-4 * 1e-3)
    assert bench.at_equal(sweep, "v", "e", mid) == pytest.approx(np.sqrt(200.0 * 400.0))
    # outside the measured range there is no number
    assert bench.at_equal(sweep, "v", "e", 5e-5) is None
    assert bench.at_equal(sweep, "v", "e", 2e-3) is None


def test_workload_names_the_configuration():
    import types
    import bench
    a = types.SimpleNamespace(n=1 << 24, theta=0.6, eps=0.005, nleaf=16, ncrit=64, level_split=5, dt=1.0 / 128,
                              seed=19810614)
    w = bench.workload(a)
    assert "N=16777216" in w and "theta=0.6" in w and "dt=1/128" in w and "FP32" in w
