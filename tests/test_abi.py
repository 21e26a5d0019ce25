"""The C ABI library loads and exports every entry point that
include/bonsai_b200.h declares; without a GPU, creating a handle fails with
an error code (no CPU fallback).  No compute calls here."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "bonsai_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(bonsai_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol(lib):
    from bonsai2_b200 import _lib
    names = declared_symbols()
    assert len(names) >= 25
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(l.split()[-1] for l in out.splitlines() if l.strip())
    missing = [s for s in names if s not in exported]
    assert not missing, missing
    for s in names:
        assert hasattr(lib, s)
    assert set(names) == set(_lib.SIGNATURES)


def test_checked_library_exports_every_declared_symbol():
    from bonsai2_b200 import _lib
    assert os.path.exists(_lib.CHECKED_LIB_PATH), "python -m bonsai2_b200.build --checks"
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.CHECKED_LIB_PATH], capture_output=True, text=True).stdout
    exported = set(l.split()[-1] for l in out.splitlines() if l.strip())
    assert not [s for s in declared_symbols() if s not in exported]


def test_bounds_check_of_normal_build_needs_no_device(lib):
    count, site = ctypes.c_uint(7), ctypes.c_uint(7)
    assert lib.bonsai_bounds_check(ctypes.byref(count), ctypes.byref(site), 1) == 0
    assert count.value == 0 and site.value == 0
    assert lib.bonsai_error_string(128)


def test_library_is_built_for_sm100a_only(lib):
    # the recipe compiles for sm_100a alone; common.cuh refuses to compile
    # device code for any other target, so a library that built is sm_100a
    from bonsai2_b200 import build
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]
    guard = open(os.path.join(ROOT, "bonsai2_b200", "csrc", "common.cuh")).read()
    assert "__CUDA_ARCH_FEAT_SM100_ALL" in guard and "#error" in guard


@pytest.mark.gpu
def test_loaded_device_code_is_sm100(lib):
    # read at run time from one of the library's own kernels
    b, p = ctypes.c_int(0), ctypes.c_int(-1)
    assert lib.bonsai_binary_version(0, ctypes.byref(b), ctypes.byref(p)) == 0
    assert b.value == 100, b.value


def test_create_without_gpu_fails_loudly(lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    import bonsai2_b200 as B
    with pytest.raises(B.BonsaiError):
        B.Treecode()


def test_error_strings(lib):
    for c in (0, -1, -2, -3, -4, -5, 1, 2, 4, 8, 16):
        assert lib.bonsai_error_string(c)


def test_default_params(lib):
    import bonsai2_b200 as B
    p = B.default_params()
    assert abs(p.theta - 0.75) < 1e-7 and abs(p.eps - 0.01) < 1e-7   # Treecode.h:164
    assert p.nleaf == 16 and p.ncrit == 64 and p.level_split == 5


def test_parameters_are_checked_before_any_device_work(lib):
    # argument errors come back before the device is touched, so they hold on any machine
    import ctypes

    import bonsai2_b200 as B
    for field, bad in (("eps", 0.0), ("eps", -1.0), ("theta", 0.0), ("nleaf", 0), ("nleaf", 65), ("ncrit", 129),
                       ("level_split", 8)):
        p = B.default_params()
        setattr(p, field, bad)
        h = ctypes.c_void_p()
        assert lib.bonsai_create(ctypes.byref(p), ctypes.byref(h)) == -4, (field, bad)
        assert not h.value
