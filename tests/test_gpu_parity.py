"""GPU parity: the CUDA path (through the C ABI) against the oracle.

Bit-exact: box, tree keys and their sort order, PH keys and order, octree
topology (canonical form: cells level by level in key order; the particle
set of every leaf), leaf list, level ranges, groups, and the walk's
interaction counts given the same cells.  Within stated tolerances:
multipoles (vs exact FP64 moments), forces (vs the FP64 direct sum, the
metric's median |da|/|a| <= 1e-3), the leapfrog update and the FP64 energy
sums.  Configuration of the small Plummer case: N=65536, seed 19810614,
theta=0.4, eps=0.01, NLEAF=16, NCRIT=64, levelSplit=5, dt=1/64.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N0 = 65536
THETA, EPS, NLEAF, NCRIT, LS, DT = 0.4, 0.01, 16, 64, 5, 1.0 / 64


def run_stages(pos, vel, theta=THETA, eps=EPS, nleaf=NLEAF, ncrit=NCRIT, ls=LS, dt=DT):
    import bonsai2_b200 as B
    t = B.Treecode(eps=eps, theta=theta, ncrit=ncrit, nleaf=nleaf, level_split=ls, dt=dt)
    t.alloc(pos.shape[0])
    t.h_ptclPos[:] = pos
    t.h_ptclVel[:] = vel
    t.ptcl_h2d()
    t.buildTree(nleaf)
    t.computeMultipoles()
    t.makeGroups(ls, ncrit)
    stats = t.computeForces(True)
    return t, stats


@pytest.fixture(scope="module")
def plummer_case(oracle, lib):
    pos, vel = oracle.plummer_float4(N0)
    t, stats = run_stages(pos, vel)
    S = oracle.OracleStep(pos, theta=THETA, eps=EPS, nleaf=NLEAF, ncrit=NCRIT, level_split=LS)
    S.build().multipoles().groups()
    return {"pos": pos, "vel": vel, "t": t, "stats": stats, "S": S, "keys": t.keys(), "cells": t.cells(),
            "groups": t.groups(), "walk": t.walk_arrays()}


def test_box_bit_exact(plummer_case):
    assert np.array_equal(plummer_case["t"].box(), plummer_case["S"].box)


def test_tree_keys_and_order_bit_exact(plummer_case, oracle):
    S, k = plummer_case["S"], plummer_case["keys"]
    ok = oracle.tree_keys(plummer_case["pos"], S.box)
    perm = oracle.argsort_u64(ok)
    assert np.array_equal(k["ids_at_build"], np.arange(N0))
    assert np.array_equal(k["tree_keys"], ok[perm])
    assert np.array_equal(k["tree_perm"], perm)


def test_ph_keys_and_order_bit_exact(plummer_case, oracle):
    S, k = plummer_case["S"], plummer_case["keys"]
    ok = oracle.ph_keys(plummer_case["pos"], S.box)
    assert np.array_equal(k["ph_keys"], S.ph_sorted)
    assert np.array_equal(k["ph_perm"], S.ph_perm)
    assert np.array_equal(np.sort(ok), k["ph_keys"])


def test_octree_topology_bit_exact(plummer_case):
    S, c, k = plummer_case["S"], plummer_case["cells"], plummer_case["keys"]
    T = S.tree
    info = c["info"]
    assert info["ncells"] == T.ncells
    assert info["nlevels"] == T.nlevels
    assert np.array_equal(info["level_beg"][1:T.nlevels + 1], T.level_beg[1:T.nlevels + 1])
    assert np.array_equal(info["level_end"][1:T.nlevels + 1], T.level_end[1:T.nlevels + 1])
    # CellData packing identical (reference layout Treecode.h:45-89)
    assert np.array_equal(c["cell_data"], T.cell_data())
    par = np.where(T.parent < 0, -1, T.parent)
    assert np.array_equal(c["parent"], par)
    # leaves: same particle sets
    tp = k["tree_perm"]
    leaf = T.nchild == 0
    for ci in np.nonzero(leaf)[0]:
        b, e = T.pbeg[ci], T.pend[ci]
        assert np.array_equal(np.sort(tp[b:e]), np.sort(T.perm[b:e]))
    # leaf list in cell order (collect_leaves, buildTree.cu:806-841)
    assert np.array_equal(c["leaf_list"], np.nonzero(leaf)[0])


def test_multipoles_vs_fp64(plummer_case, oracle):
    S, c = plummer_case["S"], plummer_case["cells"]
    T = S.tree
    ex = oracle.multipoles_fp64(T.pbeg, T.pend, plummer_case["walk"]["jpos"])
    m = c["mono"]
    assert np.allclose(m[:, 3], ex[:, 0], rtol=2e-7, atol=0)
    h = (ex[:, 13:16] - ex[:, 10:13]).max(axis=1)  # cell extent
    assert np.all(np.abs(m[:, :3] - ex[:, 1:4]).max(axis=1) <= 1e-6 * np.abs(ex[:, 1:4]).max(axis=1) + 1e-7)
    q = np.concatenate([c["quad0"], c["quad1"]], axis=1)  # xx yy zz xy xz yz
    qe = ex[:, 4:10]
    scale = np.maximum(h * h, 1e-30)
    assert np.all(np.abs(q - qe).max(axis=1) <= 1e-5 * scale + 1e-12)
    # cellOp^2 from the same definition (computeMultipoles.cu:168-177)
    cv = 0.5 * (ex[:, 13:16] + ex[:, 10:13])
    s = np.linalg.norm(cv - ex[:, 1:4], axis=1)
    l = np.maximum(2 * 0.5 * (ex[:, 13:16] - ex[:, 10:13]).max(axis=1), 1e-6)
    op2 = (l / THETA + s) ** 2
    assert np.allclose(c["size"][:, 3], op2, rtol=1e-5)
    # the reference's own arithmetic (float products, double sums) agrees too
    assert np.allclose(c["size"][:, 3], S.size4[:, 3], rtol=1e-4)


def test_groups_bit_exact(plummer_case):
    S, g = plummer_case["S"], plummer_case["groups"]
    assert np.array_equal(g[:, 0], S.gbeg)
    assert np.array_equal(g[:, 1], S.gnp)
    assert g[:, 1].sum() == N0
    # the state was gathered into PH order
    w = plummer_case["walk"]
    assert np.array_equal(w["ids"], S.ph_perm)
    assert np.array_equal(w["ipos"], S.ipos)


def test_walk_interaction_lists_exact(plummer_case, oracle):
    # the oracle walk fed with the GPU's cells and groups takes the same
    # decisions bit for bit, so interaction counts agree exactly
    S, c, g, w = plummer_case["S"], plummer_case["cells"], plummer_case["groups"], plummer_case["walk"]
    info = c["info"]
    acc, na, nd = oracle.walk(g[:, 0].copy(), g[:, 1].copy(), w["ipos"], c["cell_data"], c["size"], c["mono"],
                              c["quad0"], c["quad1"], int(info["level_beg"][1]), int(info["level_end"][1]),
                              w["jpos"], EPS)
    stats = plummer_case["stats"]
    np_ = g[:, 1].astype(np.int64)
    assert abs(stats[0] - (nd * np_).sum() / N0) < 1e-9   # <direct>
    assert abs(stats[2] - (na * np_).sum() / N0) < 1e-9   # <approx>
    assert stats[1] == nd.max() and stats[3] == na.max()
    ga = w["acc"].astype(np.float64)
    oa = acc.astype(np.float64)
    rel = np.linalg.norm(ga[:, :3] - oa[:, :3], axis=1) / np.linalg.norm(oa[:, :3], axis=1)
    assert np.percentile(rel, 99) < 2e-5
    assert np.max(np.abs(ga[:, 3] - oa[:, 3]) / np.abs(oa[:, 3])) < 2e-5


def test_forces_vs_fp64_direct_sum(plummer_case, oracle):
    # metric condition: median |da|/|a| <= 1e-3 vs the FP64 direct sum
    t = plummer_case["t"]
    acc = t.get_acc().astype(np.float64)
    rng = np.random.default_rng(7)
    samp = rng.choice(N0, 1024, replace=False)
    d = oracle.direct_fp64(plummer_case["pos"], samp, EPS, include_self=True)
    err = np.linalg.norm(acc[samp, :3] - d[:, :3], axis=1) / np.linalg.norm(d[:, :3], axis=1)
    assert np.median(err) < 1e-3
    assert np.percentile(err, 99) < 1e-2
    perr = np.abs(acc[samp, 3] - d[:, 3]) / np.abs(d[:, 3])
    assert np.median(perr) < 1e-4
    # the GPU FP64 checker agrees with the CPU one
    dg = t.direct_fp64(samp, include_self=True)
    assert np.allclose(dg, d, rtol=1e-10, atol=1e-12)


def test_leapfrog_and_energies(plummer_case, oracle):
    t = plummer_case["t"]
    pos, vel = plummer_case["pos"].copy(), plummer_case["vel"].copy()
    acc = t.get_acc()
    e_gpu = t.computeEnergies()
    t.moveParticles()
    e_gpu2 = t.computeEnergies()
    assert np.allclose(e_gpu, e_gpu2, rtol=1e-12)
    p2 = np.empty_like(pos)
    v2 = np.empty_like(vel)
    from bonsai2_b200.treecode import _p
    rc = t._L.bonsai_get_particles(t.handle, _p(p2), _p(v2), None)
    assert rc == 0
    e_or = oracle.move(pos, vel, acc, DT, False, EPS)
    assert np.array_equal(p2[:, :3], pos[:, :3])
    assert np.array_equal(v2[:, :3], vel[:, :3])
    assert np.allclose(e_gpu, e_or, rtol=1e-9, atol=1e-15)
    assert abs(e_or[7] - 1.0) < 1e-6


def test_graph_step_equals_eager_and_is_deterministic(oracle, lib):
    import bonsai2_b200 as B
    pos, vel = oracle.plummer_float4(20000)
    outs = []
    for graph in (False, True, True):
        t = B.Treecode(eps=EPS, theta=THETA, ncrit=NCRIT, nleaf=NLEAF, level_split=LS, dt=DT)
        t.alloc(pos.shape[0])
        t.h_ptclPos[:] = pos
        t.h_ptclVel[:] = vel
        t.ptcl_h2d()
        t.step(3, graph=graph)
        assert t.synchronize() == 0
        t.ptcl_d2h()
        outs.append((t.h_ptclPos.copy(), t.h_ptclVel.copy(), t.get_acc(), t.computeEnergies()))
        t.close()
    for o in outs[1:]:
        for a, b in zip(outs[0], o):
            assert np.array_equal(a, b)


def test_eager_api_step_matches_step_call(oracle, lib):
    import bonsai2_b200 as B
    pos, vel = oracle.plummer_float4(8192)
    t1, _ = run_stages(pos, vel)
    t1.moveParticles()
    t1.ptcl_d2h()
    t2 = B.Treecode(eps=EPS, theta=THETA, ncrit=NCRIT, nleaf=NLEAF, level_split=LS, dt=DT)
    t2.alloc(pos.shape[0])
    t2.h_ptclPos[:] = pos
    t2.h_ptclVel[:] = vel
    t2.ptcl_h2d()
    t2.step(1, graph=True)
    t2.ptcl_d2h()
    assert np.array_equal(t1.h_ptclPos, t2.h_ptclPos)
    assert np.array_equal(t1.h_ptclVel, t2.h_ptclVel)
