"""Regenerates the golden fixtures in tests/golden/ from the reference itself.

Only the reference's Plummer generator (code/plummer.h) runs on the CPU; it is
compiled unmodified from the reference tree by oracle/build_ref.sh into
oracle/_ref/ref_plummer and run here.  Writes:
  plummer_ref_1024.bin   full output (mass, pos, vel as FP64) for N=1024
  plummer_ref.json       sha256 of the FP64 output for several N and seeds
Run from the repository root:  python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import subprocess
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
OUT = os.path.join(ROOT, "tests", "golden")
CASES = [(1024, 19810614), (65536, 19810614), (4096, 1), (100000, 12345)]


def run_ref(n, seed):
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_plummer")
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "out.bin")
        subprocess.check_call([exe, str(n), str(seed), out], cwd=d, stdout=subprocess.DEVNULL)
        return np.fromfile(out, np.float64)


def main():
    subprocess.check_call(["sh", os.path.join(ROOT, "oracle", "build_ref.sh")])
    meta = {"source": "code/plummer.h of the reference, compiled by oracle/build_ref.sh",
            "layout": "float64: mass[n], pos[n][3], vel[n][3]", "cases": []}
    for n, seed in CASES:
        a = run_ref(n, seed)
        meta["cases"].append({"n": n, "seed": seed, "sha256": hashlib.sha256(a.tobytes()).hexdigest()})
        if n == 1024:
            a.tofile(os.path.join(OUT, "plummer_ref_1024.bin"))
    with open(os.path.join(OUT, "plummer_ref.json"), "w") as f:
        json.dump(meta, f, indent=1)


if __name__ == "__main__":
    main()
