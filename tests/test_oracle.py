"""CPU tests of the oracle (the CPU restatement of the reference algorithm):
pinned against the reference's own Plummer generator, and checked for the
internal consistency the reference's debug checks assert (every particle in
exactly one leaf, sum of group sizes = N, permutation consistency)."""
import hashlib
import json
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _gold_cases():
    with open(os.path.join(GOLD, "plummer_ref.json")) as f:
        return json.load(f)["cases"]


@pytest.mark.parametrize("case", _gold_cases(), ids=lambda c: "n%d_s%d" % (c["n"], c["seed"]))
def test_plummer_matches_reference_generator(oracle, case):
    # code/plummer.h:9-138 run unmodified -> sha256 fixture
    m, p, v = oracle.plummer(case["n"], case["seed"])
    a = np.concatenate([m, p.ravel(), v.ravel()])
    assert hashlib.sha256(a.tobytes()).hexdigest() == case["sha256"]


def test_plummer_full_vector_1024(oracle):
    ref = np.fromfile(os.path.join(GOLD, "plummer_ref_1024.bin"), np.float64)
    m, p, v = oracle.plummer(1024, 19810614)
    assert np.array_equal(ref, np.concatenate([m, p.ravel(), v.ravel()]))
    assert abs(m.sum() - 1.0) < 1e-12


def test_product_plummer_matches_oracle(oracle, lib):
    # the product's host IC generator (libbonsai_b200.so) reproduces the same stream
    import bonsai2_b200 as B
    for n, seed in [(1024, 19810614), (4096, 1)]:
        p, v = B.plummer(n, seed)
        po, vo = oracle.plummer_float4(n, seed)
        assert np.array_equal(p, po) and np.array_equal(v, vo)


def _pos(oracle, n, seed=19810614):
    p, v = oracle.plummer_float4(max(n, 64), seed)
    return np.ascontiguousarray(p[:n]), np.ascontiguousarray(v[:n])


@pytest.mark.parametrize("n,nleaf", [(1, 16), (10, 16), (17, 16), (3000, 16), (20000, 24), (20000, 64), (8192, 1)])
def test_tree_partition_properties(oracle, n, nleaf):
    p, _ = _pos(oracle, n)
    box, bad = oracle.bbox(p)
    assert bad == 0
    t = oracle.OracleTree(p, box, nleaf)
    # permutation is a bijection; every particle in exactly one leaf
    assert np.array_equal(np.sort(t.perm), np.arange(n))
    leaf = t.nchild == 0
    assert (t.pend[leaf] - t.pbeg[leaf]).sum() == n
    assert np.all(t.pend[leaf] - t.pbeg[leaf] <= nleaf) or t.overflow
    assert np.all(t.pend[~leaf] - t.pbeg[~leaf] > nleaf)
    # children contiguous, one level down, and cover the parent range
    for c in np.nonzero(~leaf)[0]:
        f, k = t.first[c], t.nchild[c]
        assert np.all(t.level[f:f + k] == t.level[c] + 1)
        assert np.all(t.parent[f:f + k] == c)
        assert t.pbeg[f] == t.pbeg[c] and t.pend[f + k - 1] == t.pend[c]
    # level ranges
    for L in range(1, t.nlevels + 1):
        assert np.all(t.level[t.level_beg[L]:t.level_end[L]] == L)
    # every particle lies in its leaf's box: the octant path keys agree
    keys = oracle.tree_keys(p, box)
    for c in np.nonzero(leaf)[0][:200]:
        sh = np.uint64(63 - 3 * int(t.level[c]))
        pre = keys[t.perm[t.pbeg[c]:t.pend[c]]] >> sh
        assert np.all(pre == pre[0])


def test_key_order_reproduces_comparison_partition(oracle):
    # sorting the exact octant-path keys groups every cell contiguously in the
    # same cell order as the breadth-first comparison partition
    p, _ = _pos(oracle, 30000)
    box, _ = oracle.bbox(p)
    t = oracle.OracleTree(p, box, 16)
    k = oracle.tree_keys(p, box)
    perm = oracle.argsort_u64(k)
    for c in range(t.ncells):
        b, e = t.pbeg[c], t.pend[c]
        assert np.array_equal(np.sort(perm[b:e]), np.sort(t.perm[b:e]))


def test_argsort_stable(oracle):
    rng = np.random.default_rng(3)
    k = rng.integers(0, 50, 10000).astype(np.uint64) << np.uint64(40)
    perm = oracle.argsort_u64(k)
    assert np.array_equal(perm, np.argsort(k, kind="stable"))


def test_groups_properties(oracle):
    p, _ = _pos(oracle, 50000)
    box, _ = oracle.bbox(p)
    k = oracle.ph_keys(p, box)
    ks = k[oracle.argsort_u64(k)]
    for ls, nc in [(1, 64), (5, 64), (5, 32), (7, 128)]:
        gb, gn = oracle.make_groups(ks, ls, nc)
        assert gn.sum() == p.shape[0]
        assert np.all(gn >= 1) and np.all(gn <= nc)
        assert np.array_equal(gb[1:], gb[:-1] + gn[:-1])
        mask_shift = np.uint64(63 - 3 * ls)
        for g in range(0, len(gb), 97):
            seg = ks[gb[g]:gb[g] + gn[g]] >> mask_shift
            assert np.all(seg == seg[0])


def test_walk_against_direct_sum(oracle):
    # median |da|/|a| of the reference algorithm at theta=0.4 vs FP64 direct sum
    n = 8192
    p, _ = _pos(oracle, n)
    S = oracle.OracleStep(p, theta=0.4, eps=0.01).build().multipoles().groups().forces()
    rng = np.random.default_rng(1)
    samp = rng.choice(n, 256, replace=False)
    d = oracle.direct_fp64(p, S.ph_perm[samp], 0.01)
    a = S.acc[samp].astype(np.float64)
    err = np.linalg.norm(a[:, :3] - d[:, :3], axis=1) / np.linalg.norm(d[:, :3], axis=1)
    assert np.median(err) < 1e-3
    perr = np.abs(a[:, 3] - d[:, 3]) / np.abs(d[:, 3])
    assert np.median(perr) < 1e-4


def test_leapfrog_energy_drift(oracle):
    # KDK with merged kicks conserves energy to O(dt^2) on a small Plummer sphere
    n = 2048
    p, v = _pos(oracle, n)
    eps, dt = 0.05, 1.0 / 128
    E = []
    closing = False
    for step in range(8):
        S = oracle.OracleStep(p, theta=0.3, eps=eps).build().multipoles().groups().forces()
        acc = np.empty_like(S.acc)
        acc[S.ph_perm] = S.acc
        e = oracle.move(p, v, acc, dt, closing, eps)
        closing = True
        E.append(e[3])
    E = np.array(E)
    assert abs(E[-1] - E[0]) / abs(E[0]) < 1e-3


def test_multipoles_ref_vs_fp64(oracle):
    p, _ = _pos(oracle, 20000)
    S = oracle.OracleStep(p, theta=0.4, eps=0.01).build().multipoles()
    t = S.tree
    ex = oracle.multipoles_fp64(t.pbeg, t.pend, S.jpos)
    assert np.allclose(S.mono4[:, 3], ex[:, 0], rtol=1e-6)
    assert np.allclose(S.mono4[:, :3], ex[:, 1:4], rtol=1e-5, atol=1e-6)


def test_oracle_tree_shape_matches_the_published_build(oracle):
    """treebuild/readme:33-39: the reference's build of a float32 Plummer sphere
    (plummer.h, default seed), N = 20,000,000, NLEAF 16, has 596,463 nodes,
    4,041,848 leaves, 4,638,311 cells and 15 levels.  The oracle's comparison
    partition reproduces it exactly (about 10 s on 8 cores)."""
    pos, _ = oracle.plummer_float4(20_000_000, 19810614)
    box, _ = oracle.bbox(pos)
    T = oracle.OracleTree(pos, box, 16)
    assert T.ncells == 4638311
    assert int((T.nchild > 0).sum()) == 596463
    assert int((T.nchild == 0).sum()) == 4041848
    assert int(T.level.max()) == 15
