"""Regenerates tests/golden/ref_groups.json from the reference's own GPU group
formation (Treecode<float>::makeGroups, code/makeGroups.cu, compiled unmodified
for sm_100a by oracle/build_ref.sh into oracle/_ref/ref_groups).

Needs a GPU (the reference's kernels and Thrust sort run on it) and the binary
built beforehand; it does not rebuild it.  For each case the input is made by
the oracle's Plummer generator (pinned to code/plummer.h) or a seeded numpy
draw, the domain box by the oracle's restatement of computeBoundingBox
(buildTree.cu:80-166, which does not build for sm_100), and the reference then
computes the PH keys, sorts them with Thrust and forms the groups.  Recorded:
sha256 of the full 63-bit PH keys in input order (uint64, from the reference's
computeKeys<21> launched alone), of the sorted keys as makeGroups leaves them
(masked to the top levelSplit digits by mask_keys), of the sort permutation
(int32) and of the group list ordered by first particle (int32 pairs; the
reference numbers groups in atomicAdd order), the group count, and for the
first case the whole list.

usage (repository root, on a GPU machine):
    python tests/golden/make_ref_groups.py [OUT.json]
"""
import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

# (name, generator, n, seed, level_split, ncrit)
CASES = [
    ("plummer_65536", "plummer", 65536, 19810614, 5, 64),
    ("plummer_1000000", "plummer", 1000000, 12345, 5, 64),
    ("plummer_65536_coincident_2000", "plummer_coincident", 65536, 1, 3, 32),
    ("uniform_100003", "uniform", 100003, 7, 7, 17),
]


def make_input(gen, n, seed):
    """float4 (x, y, z, m) input of a case; the same function feeds the tests."""
    if gen in ("plummer", "plummer_coincident"):
        pos, _ = O.plummer_float4(n, seed)
        if gen == "plummer_coincident":
            pos[:2000, :3] = pos[0, :3]  # 2000 equal keys: the sort's tie order is on trial
        return pos
    rng = np.random.default_rng(seed)
    pos = np.empty((n, 4), np.float32)
    pos[:, :3] = rng.uniform(-1.0, 1.0, (n, 3)).astype(np.float32)
    pos[:, 3] = np.float32(1.0 / n)
    return pos


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def groups_by_pbeg(groups):
    g = np.asarray(groups, np.int32).reshape(-1, 2)
    return g[np.argsort(g[:, 0], kind="stable")]


def run_ref(pos, box, level_split, ncrit, reps=1, prefix=True):
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_groups")
    n = pos.shape[0]
    with tempfile.TemporaryDirectory() as d:
        inp = os.path.join(d, "in.f32")
        np.ascontiguousarray(pos, np.float32).tofile(inp)
        args = [exe, inp, str(n)] + ["%.9g" % float(b) for b in box] + [str(level_split), str(ncrit), str(reps)]
        if prefix:
            args.append(os.path.join(d, "out"))
        r = subprocess.run(args, capture_output=True, text=True, check=True)
        info = json.loads([l for l in r.stdout.splitlines() if l.startswith("REFGROUPS ")][-1][len("REFGROUPS "):])
        if not prefix:
            return info, None
        raw = np.fromfile(os.path.join(d, "out.rawkeys"), np.uint64)
        masked = np.fromfile(os.path.join(d, "out.keys"), np.uint64)
        vals = np.fromfile(os.path.join(d, "out.vals"), np.int32)
        groups = np.fromfile(os.path.join(d, "out.groups"), np.int32).reshape(-1, 2)
        return info, (raw, masked, vals, groups)


def level_mask(level_split):
    """makeGroups' segment mask (makeGroups.cu:259-266): the top levelSplit of 21 octal digits."""
    return np.uint64(((1 << (3 * level_split)) - 1) << (63 - 3 * level_split))


def main():
    out = sys.argv[1] if len(sys.argv) > 1 else os.path.join(ROOT, "tests", "golden", "ref_groups.json")
    meta = {"source": "code/makeGroups.cu of the reference (PH keys, Thrust sort_by_key, segment scans, groups), "
                      "compiled unmodified for sm_100a by oracle/build_ref.sh, run on a B200",
            "box": "oracle.bbox (restates buildTree.cu:80-166)", "cases": []}
    for name, gen, n, seed, ls, nc in CASES:
        pos = make_input(gen, n, seed)
        box, bad = O.bbox(pos)
        assert not bad
        info, (raw, masked, vals, groups) = run_ref(pos, box, ls, nc)
        assert np.array_equal(masked, raw[vals] & level_mask(ls))  # the reference's own outputs agree
        g = groups_by_pbeg(groups)
        case = {"name": name, "generator": gen, "n": n, "seed": seed, "level_split": ls, "ncrit": nc,
                "box": [float(b) for b in box], "ngroups": int(g.shape[0]),
                "sha256_keys": sha(raw), "sha256_masked_sorted_keys": sha(masked), "sha256_perm": sha(vals),
                "sha256_groups_by_pbeg": sha(g)}
        if name == "plummer_65536":
            case["groups_by_pbeg"] = g.tolist()
        meta["cases"].append(case)
        print(name, info, flush=True)
    with open(out, "w") as f:
        json.dump(meta, f, indent=1)
        f.write("\n")
    print("wrote", out)


if __name__ == "__main__":
    main()
