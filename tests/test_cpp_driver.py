"""The header-only C++ Treecode<float> (include/bonsai_treecode.hpp) compiles
against a driver shaped like the reference's treecode.cu and links with
libbonsai_b200.so.  Without a GPU the driver must fail with
BONSAI_ERR_NO_DEVICE (no CPU fallback); with one it runs a full step."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def driver(lib, tmp_path_factory):
    out = str(tmp_path_factory.mktemp("drv") / "driver")
    libdir = os.path.join(ROOT, "bonsai2_b200")
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
                           os.path.join(ROOT, "tests", "cpp", "driver.cpp"), "-L", libdir, "-lbonsai_b200",
                           "-Wl,-rpath," + libdir, "-o", out])
    return out


def test_driver_builds_and_reports_no_device(driver):
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    r = subprocess.run([driver, "1024"], capture_output=True, text=True)
    assert r.returncode == 3, r.stdout + r.stderr


@pytest.mark.gpu
def test_driver_runs_a_step(driver):
    r = subprocess.run([driver, "8192"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("ok n=8192")
    fields = dict(kv.split("=") for kv in r.stdout.split()[1:])
    assert float(fields["direct"]) > 0 and float(fields["approx"]) > 0
    assert abs(float(fields["M"]) - 1.0) < 1e-6
