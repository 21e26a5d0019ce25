"""The bounds-checked build (libbonsai_b200_checks.so, -DBONSAI_CHECKS).

compute-sanitizer is not available for these runs, so the library carries its
own checks: every guarded kernel index (cells, leaves, groups, particles,
scatter destinations) is tested, and an out-of-range one is counted and its
access skipped.  The checked library runs the workloads of
tests/checked_workload.py in a child process (the library is chosen per
process); every case must finish with its expected status and no violation.
The overflow cases show that the capacity guards stop every write before the
arrays' ends: the cell arrays outgrown in a graph replay and a walk level list
outgrown at a tiny opening angle report their status bits and nothing else."""
import ctypes
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _checked_lib():
    from bonsai2_b200 import _lib
    path = _lib.CHECKED_LIB_PATH
    assert os.path.exists(path), "bounds-checked library missing: python -m bonsai2_b200.build --checks"
    return path


def test_selftest_counts_in_checked_build_only():
    import bonsai2_b200 as B
    assert B.load().bonsai_bounds_selftest(0) == 0
    assert B.bounds_check() == {"checked": False, "count": 0, "first_site": 0}
    lib = ctypes.CDLL(_checked_lib())
    lib.bonsai_bounds_selftest.argtypes = [ctypes.c_int]
    assert lib.bonsai_bounds_selftest(0) == 1
    count, site = ctypes.c_uint(0), ctypes.c_uint(0)
    lib.bonsai_bounds_check.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
    assert lib.bonsai_bounds_check(ctypes.byref(count), ctypes.byref(site), 1) == 1
    assert count.value == 1 and site.value == 0x7FF
    assert lib.bonsai_bounds_check(ctypes.byref(count), ctypes.byref(site), 0) == 1 and count.value == 0


def test_workloads_in_bounds():
    env = dict(os.environ, BONSAI_B200_LIB=_checked_lib())
    r = subprocess.run([sys.executable, os.path.join(ROOT, "tests", "checked_workload.py")], env=env,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert out["checked"] and out["selftest"] == 1
    expected_status = {
        "case_plummer": [0, 0],
        "case_leaf_and_group_sizes": [0, 0, 0, 0, 0],
        "case_ensemble": [0, 0, 0],
        "case_double_single": [0, 0],
        "case_block_steps": [0],
        "case_per_group_theta": [0, 0],
        "case_cell_capacity_overflow": [0, 1],
        "case_walk_list_overflow": [4],
        "case_coincident": [2],
    }
    for name, want in expected_status.items():
        got = out[name]
        assert got["violations"] == 0, f"{name}: {got['violations']} out-of-range indexes, first site {got['first_site']:#x}"
        assert got["status"] == want, f"{name}: status {got['status']}"
