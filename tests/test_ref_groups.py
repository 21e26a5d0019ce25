"""The oracle's PH keys, sort order and groups against the reference's own GPU
group formation (code/makeGroups.cu run unmodified on a B200; fixtures in
tests/golden/ref_groups.json, made by tests/golden/make_ref_groups.py).

Four cases: Plummer N = 65,536 and 1,000,000 at levelSplit 5 / nCrit 64, a
Plummer sphere with 2,000 coincident particles (equal keys: the stable tie
order of Thrust's sort) at levelSplit 3 / nCrit 32, and a uniform cube of
100,003 particles at levelSplit 7 / nCrit 17.  Bit-exact: the full 63-bit keys,
the sorted keys as the reference leaves them (masked to the top levelSplit
digits), the permutation and the group list."""
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))

from make_ref_groups import groups_by_pbeg, level_mask, make_input, sha  # noqa: E402

CASES = json.load(open(os.path.join(ROOT, "tests", "golden", "ref_groups.json")))["cases"]


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_oracle_matches_reference_make_groups(case):
    from oracle import oracle as O
    pos = make_input(case["generator"], case["n"], case["seed"])
    box, bad = O.bbox(pos)
    assert not bad and [float(b) for b in box] == case["box"]
    keys = O.ph_keys(pos, box)
    perm = O.argsort_u64(keys)
    sk = keys[perm]
    gb, gn = O.make_groups(sk, case["level_split"], case["ncrit"])
    g = groups_by_pbeg(np.stack([gb, gn], 1))
    assert sha(keys) == case["sha256_keys"]
    assert sha(sk & level_mask(case["level_split"])) == case["sha256_masked_sorted_keys"]
    assert sha(perm) == case["sha256_perm"]
    assert g.shape[0] == case["ngroups"] and sha(g) == case["sha256_groups_by_pbeg"]
    if "groups_by_pbeg" in case:
        assert np.array_equal(g, np.asarray(case["groups_by_pbeg"], np.int32))
