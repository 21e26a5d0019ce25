"""The library's PH keys, sort order and groups against the reference's own GPU
group formation (code/makeGroups.cu run unmodified on a B200; fixtures in
tests/golden/ref_groups.json, made by tests/golden/make_ref_groups.py; the
same four cases as tests/test_ref_groups.py).  Bit-exact."""
import json
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))

from make_ref_groups import groups_by_pbeg, level_mask, make_input, sha  # noqa: E402

CASES = json.load(open(os.path.join(ROOT, "tests", "golden", "ref_groups.json")))["cases"]


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_library_matches_reference_make_groups(case):
    import bonsai2_b200 as B
    pos = make_input(case["generator"], case["n"], case["seed"])
    n = pos.shape[0]
    t = B.Treecode(eps=0.01, theta=0.5, ncrit=case["ncrit"], level_split=case["level_split"])
    t.alloc(n)
    t.h_ptclPos[:] = pos
    t.h_ptclVel[:] = 0.0
    t.ptcl_h2d()
    t.buildTree(16)
    t.makeGroups(case["level_split"], case["ncrit"])
    assert t.synchronize() in (0, 2)  # 2: coincident particles past depth 21 (a fat leaf; the groups are unaffected)
    assert [float(b) for b in t.box()] == case["box"]
    k = t.keys()
    assert np.array_equal(k["ids_at_build"], np.arange(n))
    perm, sk = k["ph_perm"], k["ph_keys"]
    keys = np.empty(n, np.uint64)
    keys[perm] = sk
    assert sha(keys) == case["sha256_keys"]
    assert sha(sk & level_mask(case["level_split"])) == case["sha256_masked_sorted_keys"]
    assert sha(perm) == case["sha256_perm"]
    g = groups_by_pbeg(t.groups())
    assert g.shape[0] == case["ngroups"] and sha(g) == case["sha256_groups_by_pbeg"]
    t.close()
