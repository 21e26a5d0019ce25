"""Build recipe of libbonsai_b200.so (in-tree, sm_100a).

nvcc compiles every .cu in bonsai2_b200/csrc for sm_100a only; the tree walk
translation unit flushes denormals (-ftz=true) like the reference's
computeForces.o rule (code/Makefile:53-54).  Objects go to
bonsai2_b200/_build/, the library to bonsai2_b200/libbonsai_b200.so.
`--checks` builds the bounds-checked variant (-DBONSAI_CHECKS: every guarded
kernel index is tested and counted instead of accessed out of range) into
bonsai2_b200/libbonsai_b200_checks.so, objects in bonsai2_b200/_build_checks/.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libbonsai_b200.so")
# bounds-checked variant (-DBONSAI_CHECKS): every guarded kernel index tested
LIB_CHECKS = os.path.join(HERE, "libbonsai_b200_checks.so")
OBJ_CHECKS = os.path.join(HERE, "_build_checks")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I", INCLUDE, "--expt-relaxed-constexpr"]
# extra -D tuning flags (e.g. BONSAI_WALK_SPLIT=0) for alternative builds
EXTRA = os.environ.get("BONSAI_NVCC_DEFINES", "").split()
PER_FILE = {"walk.cu": ["-ftz=true"], "walk64.cu": ["-ftz=true"]}
SOURCES = ["keys.cu", "sort.cu", "tree.cu", "multipoles.cu", "groups.cu", "walk.cu", "move.cu", "treecode.cu",
           "noalloc.cu", "learned.cu", "walk64.cu"]
HOST_SOURCES = ["plummer.cpp", "ics.cpp", "tipsy.cpp"]


def _deps():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(INCLUDE, "bonsai_b200.h")]


def up_to_date(lib: str = LIB) -> bool:
    if not os.path.exists(lib):
        return False
    t = os.path.getmtime(lib)
    return all(os.path.getmtime(d) <= t for d in _deps())


def _compile(src: str, verbose: bool, objdir: str, extra: list) -> str:
    out = os.path.join(objdir, src + ".o")
    path = os.path.join(CSRC, src)
    if src.endswith(".cpp"):
        cmd = ["g++", "-O3", "-fPIC", "-std=c++17", "-c", path, "-o", out]
    else:
        cmd = [NVCC] + ARCH + COMMON + EXTRA + extra + PER_FILE.get(src, []) + (["-Xptxas", "-v"] if verbose else []) + ["-c", path, "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("compile failed: %s\n%s\n%s" % (" ".join(cmd), r.stdout, r.stderr))
    if verbose:
        sys.stderr.write(r.stderr)
    return out


def build(force: bool = False, verbose: bool = False, out: str = None, objdir: str = None,
          checks: bool = False) -> str:
    """Builds the library (checks: the bounds-checked variant) and returns its path."""
    default = LIB_CHECKS if checks else LIB
    lib = out or default
    if not force and out is None and up_to_date(default):
        return default
    objdir = objdir or (OBJ_CHECKS if checks else OBJ)
    extra = ["-DBONSAI_CHECKS"] if checks else []
    os.makedirs(objdir, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose, objdir, extra), SOURCES + HOST_SOURCES))
    tmp = lib + ".tmp%d" % os.getpid()
    cmd = [NVCC] + ARCH + ["-shared", "-o", tmp] + objs + ["-lcudart"]
    subprocess.check_call(cmd)
    os.replace(tmp, lib)
    return lib


if __name__ == "__main__":
    import argparse
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", action="store_true")
    ap.add_argument("--out", default=None, help="write the library here instead of the in-tree path")
    ap.add_argument("--objdir", default=None)
    ap.add_argument("--checks", action="store_true", help="the bounds-checked variant (-DBONSAI_CHECKS)")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.v, out=a.out, objdir=a.objdir, checks=a.checks))
