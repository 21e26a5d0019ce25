"""Driver of the "modified reference" walk (oracle/_ref/ref_walk).

Test and baseline infrastructure only.  The harness (oracle/ref_walk_main.cu)
runs the reference's own Treecode<float>::computeMultipoles and
Treecode<float>::computeForces (code/computeMultipoles.cu,
code/computeForces.cu, with the mechanical sm_100a shims of
oracle/make_modref.py) on a tree that the library built; this module writes
that tree in the harness's input format and reads the results back.  The
reference cannot build its own tree on sm_100 (buildTree.cu needs
CUDA-12-removed device synchronisation), so the cells, level-1 range and
groups are the library's, exported in the reference's layout.
"""
from __future__ import annotations

import json
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
EXE = os.path.join(HERE, "_ref", "ref_walk")
MAGIC = 0x4B4C5752


def available() -> bool:
    return os.access(EXE, os.X_OK)


def tree_of(t) -> dict:
    """The walk inputs of a library handle after computeMultipoles and
    makeGroups: cells in the reference's layout, level-1 range, groups, and
    the i- (group order) and j- (tree order) particle arrays."""
    c = t.cells(multipoles=True)
    info = c["info"]
    w = t.walk_arrays()
    return {"cell_data": c["cell_data"], "size": c["size"], "mono": c["mono"], "quad0": c["quad0"],
            "quad1": c["quad1"], "l1": (int(info["level_beg"][1]), int(info["level_end"][1])),
            "groups": t.groups(), "ipos": w["ipos"], "jpos": w["jpos"], "acc": w["acc"]}


def write_input(path: str, tree: dict, theta: float, eps2: float, ncrit: int) -> None:
    n = tree["ipos"].shape[0]
    hdr = np.array([MAGIC, n, tree["cell_data"].shape[0], tree["groups"].shape[0], tree["l1"][0], tree["l1"][1],
                    ncrit, 0], np.int32)
    with open(path, "wb") as f:
        f.write(hdr.tobytes())
        f.write(np.array([theta, eps2], np.float32).tobytes())
        for k, dt in (("cell_data", np.uint32), ("size", np.float32), ("mono", np.float32), ("quad0", np.float32),
                      ("quad1", np.float32), ("groups", np.int32), ("ipos", np.float32), ("jpos", np.float32)):
            f.write(np.ascontiguousarray(tree[k], dt).tobytes())


def _line(stdout: str, tag: str) -> dict:
    for ln in stdout.splitlines():
        if ln.startswith(tag + " "):
            return json.loads(ln[len(tag) + 1:])
    raise RuntimeError("ref_walk printed no %s line" % tag)


def check(inp: str, prefix: str, ncells: int, ngroups: int, n: int, timeout: float = 600) -> dict:
    """Reference multipoles of the tree and the reference walk with the
    library's and with its own multipoles (oracle/ref_walk_main.cu, mode
    check)."""
    r = subprocess.run([EXE, "check", inp, prefix], capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError("ref_walk check exited %d: %s" % (r.returncode, r.stderr[-2000:]))
    out = _line(r.stdout, "REFWALK")
    mp = np.fromfile(prefix + ".refmp", np.uint8)
    off = 0
    res = {"stats": out}
    for k, w in (("size", 4), ("mono", 4), ("quad0", 4), ("quad1", 2)):
        nb = ncells * w * 4
        res["ref_" + k] = mp[off:off + nb].view(np.float32).reshape(ncells, w)
        off += nb
    for k in ("lib", "ref"):
        res["acc_" + k] = np.fromfile(prefix + ".acc_" + k, np.float32).reshape(n, 4)
        res["cnt_" + k] = np.fromfile(prefix + ".cnt_" + k, np.uint32).reshape(ngroups, 2)
    return res


def time_walk(inp: str, reps: int, timeout: float = 900) -> dict:
    """computeMultipoles and computeForces timed by the harness (mode time)."""
    r = subprocess.run([EXE, "time", inp, str(reps)], capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        return {"unavailable": "ref_walk time exited %d: %s" % (r.returncode, r.stderr[-500:])}
    return _line(r.stdout, "REFWALK_TIME")
