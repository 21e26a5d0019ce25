"""Regenerates tests/golden/ref_walk.npz from the reference's own multipole
and tree-walk code (Treecode<float>::computeMultipoles and ::computeForces,
code/computeMultipoles.cu and code/computeForces.cu with the mechanical sm_100a
shims of oracle/make_modref.py, run by oracle/_ref/ref_walk).

Needs a GPU and the binary built beforehand (oracle/build_ref.sh); it does not
rebuild it.  For each case the library builds the tree (box, keys, octree,
multipoles, groups) of a Plummer sphere from the reference's own generator
(pinned to code/plummer.h), and the reference then computes its multipoles of
those cells and walks them twice: with the library's multipoles and with its
own.  Recorded per case: sha256 of the inputs the reference was given (cells,
groups, i- and j-particles), the reference's per-group interaction counts
(approximate, direct) of both walks, its accelerations (every STRIDE-th
particle in group order), its multipoles (every 4th cell) and the statistics
that computeForces returns (mean and max direct, mean and max approximate).

usage (repository root, on a GPU machine):
    python tests/golden/make_ref_walk.py [OUT.npz]
"""
import hashlib
import json
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

# (name, n, seed, theta, eps, nleaf, ncrit, level_split, acc stride)
CASES = [
    ("plummer_65536_theta04", 65536, 19810614, 0.4, 0.01, 16, 64, 5, 4),
    ("plummer_65536_theta075", 65536, 2, 0.75, 0.005, 16, 64, 5, 16),
]
CELL_STRIDE = 4


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def library_tree(case):
    """The library's tree of a case, and its own walk (the handle stays open)."""
    import bonsai2_b200 as B

    name, n, seed, theta, eps, nleaf, ncrit, ls, stride = case
    pos, vel = B.plummer(n, seed)
    t = B.Treecode(eps=eps, theta=theta, ncrit=ncrit, nleaf=nleaf, level_split=ls, dt=1.0 / 64)
    t.alloc(n)
    t.h_ptclPos[:] = pos
    t.h_ptclVel[:] = vel
    t.ptcl_h2d()
    t.buildTree(nleaf)
    t.computeMultipoles()
    t.makeGroups(ls, ncrit)
    stats = t.computeForces(True)
    assert t.synchronize() == 0
    return t, stats


def input_hashes(tree):
    return {k: sha(np.ascontiguousarray(tree[k])) for k in ("cell_data", "groups", "ipos", "jpos")}


def main(out):
    from oracle import ref_walk as RW

    if not RW.available():
        raise SystemExit("oracle/_ref/ref_walk is not built (oracle/build_ref.sh)")
    arrays, meta = {}, {}
    with tempfile.TemporaryDirectory() as tmp:
        for case in CASES:
            name, n, seed, theta, eps, nleaf, ncrit, ls, stride = case
            t, stats = library_tree(case)
            tree = RW.tree_of(t)
            t.close()
            inp = os.path.join(tmp, name + ".in")
            eps2 = float(np.float32(np.float32(eps) * np.float32(eps)))
            RW.write_input(inp, tree, theta, eps2, ncrit)
            r = RW.check(inp, os.path.join(tmp, name), tree["cell_data"].shape[0], tree["groups"].shape[0], n)
            arrays[name + "/cnt_lib"] = r["cnt_lib"]
            arrays[name + "/cnt_ref"] = r["cnt_ref"]
            arrays[name + "/acc_lib"] = r["acc_lib"][::stride]
            arrays[name + "/acc_ref"] = r["acc_ref"][::stride]
            for k in ("size", "mono", "quad0", "quad1"):
                arrays[name + "/ref_" + k] = r["ref_" + k][::CELL_STRIDE]
            meta[name] = {"case": list(case), "inputs_sha256": input_hashes(tree), "ref_stats": r["stats"],
                          "library_stats": [float(s) for s in stats], "cells": int(tree["cell_data"].shape[0]),
                          "groups": int(tree["groups"].shape[0])}
            # what the test will find, printed for the record
            ga = tree["acc"].astype(np.float64)
            ra = r["acc_lib"].astype(np.float64)
            rel = np.linalg.norm(ga[:, :3] - ra[:, :3], axis=1) / np.linalg.norm(ra[:, :3], axis=1)
            print(name, json.dumps(r["stats"]), "library stats", [round(float(s), 6) for s in stats],
                  "| acc vs reference walk (library multipoles): median %.2e p99 %.2e max %.2e" % (
                      np.median(rel), np.percentile(rel, 99), rel.max()),
                  "| groups whose counts differ between the reference walk on library and on reference "
                  "multipoles: %d of %d" % (int((r["cnt_lib"] != r["cnt_ref"]).any(axis=1).sum()),
                                            tree["groups"].shape[0]))
    arrays["meta"] = np.frombuffer(json.dumps(meta).encode(), np.uint8)
    np.savez_compressed(out, **arrays)
    print("wrote", out, os.path.getsize(out), "bytes")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(ROOT, "tests", "golden", "ref_walk.npz"))
