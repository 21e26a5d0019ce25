"""The FP64 checker walk: the float walk's interaction lists, FP64 arithmetic."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _stats(t):
    import bonsai2_b200 as B
    st = np.zeros(4, np.uint64)
    assert t._L.bonsai_get_stats(t.handle, B.treecode._p(st)) == 0
    return st


def _rel(a, b):
    return np.linalg.norm(a[:, :3] - b[:, :3], axis=1) / np.linalg.norm(b[:, :3], axis=1)


def test_same_lists_rounding_only_plummer():
    import bonsai2_b200 as B
    n = 65536
    p, v = B.plummer(n, 19810614)
    t = B.Treecode(eps=0.01, theta=0.4)
    t.alloc(n)
    t.h_ptclPos[:] = p
    t.h_ptclVel[:] = v
    t.ptcl_h2d()
    t.buildTree(16)
    t.computeMultipoles()
    t.makeGroups(5, 64)
    t.computeForces(False)
    a32 = t.get_acc().astype(np.float64)
    s32 = _stats(t)
    a64, s64 = t.compute_forces_fp64()
    assert np.array_equal(s32, s64)  # identical interaction lists
    d = _rel(a32, a64)
    assert np.median(d) < 1e-6 and np.percentile(d, 99) < 1e-5  # FP32 rounding only
    rng = np.random.default_rng(1)
    samp = np.sort(rng.choice(n, 1024, replace=False)).astype(np.int32)
    ref = t.direct_fp64(samp)
    e32, e64 = _rel(a32[samp], ref), _rel(a64[samp], ref)
    # truncation dominates: the FP64 walk's error is the float walk's to a few per cent
    assert abs(np.median(e64) / np.median(e32) - 1) < 0.05
    t.close()


def test_double_single_far_from_origin_matches_fp64():
    import bonsai2_b200 as B
    n = 16384
    p, v = B.galaxy(n, seed=6)
    p[:, :3] += np.array([1.0e4, -7.0e3, 5.0e3])
    t = B.Treecode(eps=0.01, theta=0.5)
    t.set_precision(1)
    t.set_particles_f64(p, v)
    t.buildTree(16)
    t.computeMultipoles()
    t.makeGroups(5, 64)
    t.computeForces(False)
    a_ds = t.get_acc().astype(np.float64)
    a64, s64 = t.compute_forces_fp64()
    assert np.array_equal(_stats(t), s64)
    assert np.median(_rel(a_ds, a64)) < 1e-5
    t.close()


def test_per_group_angles_in_fp64_walk():
    import bonsai2_b200 as B
    n = 32768
    p, v = B.plummer(n, 2)
    t = B.Treecode(eps=0.01, theta=0.5)
    t.alloc(n)
    t.h_ptclPos[:] = p
    t.h_ptclVel[:] = v
    t.ptcl_h2d()
    t.buildTree(16)
    t.computeMultipoles()
    t.makeGroups(5, 64)
    a_fixed, s_fixed = t.compute_forces_fp64()
    ng = t.groups().shape[0]
    assert t._L.bonsai_set_theta_mode(t.handle, 2, 0.25, 1.25) == 0
    th = np.full(ng, 0.5, np.float32)
    assert t._L.bonsai_set_group_theta(t.handle, B.treecode._p(th), ng) == 0
    a_pg, s_pg = t.compute_forces_fp64()
    assert np.array_equal(s_fixed, s_pg)
    assert np.array_equal(a_fixed.view(np.uint64), a_pg.view(np.uint64))
    t.close()


def test_fp64_walk_inside_an_ensemble_is_per_system():
    """In an ensemble every group's FP64 walk starts from its own system's
    level-1 cells: the interaction lists are the float walk's, and each
    system's FP64 forces are bit-identical to those it gets alone."""
    import bonsai2_b200 as B
    from bonsai2_b200.ensemble import plummer_ensemble
    counts = np.array([300, 1, 2000, 57, 2], np.int32)
    pos, vel = plummer_ensemble(counts, base_seed=41)
    off = np.concatenate([[0], np.cumsum(counts)])

    def run(t, p, v):
        t.h_ptclPos[:] = p
        t.h_ptclVel[:] = v
        t.ptcl_h2d()
        t.buildTree(16)
        t.computeMultipoles()
        t.makeGroups(5, 64)
        t.computeForces(False)
        s32 = _stats(t)
        a64, s64 = t.compute_forces_fp64()
        assert t.synchronize() == 0
        assert np.array_equal(s32, s64)
        return a64

    t = B.Treecode(eps=0.01, theta=0.5)
    t.set_systems(counts)
    a_ens = run(t, pos, vel)
    t.close()
    for s in range(counts.shape[0]):
        b, e = off[s], off[s + 1]
        u = B.Treecode(eps=0.01, theta=0.5)
        u.alloc(int(e - b))
        a_alone = run(u, pos[b:e], vel[b:e])
        u.close()
        assert np.array_equal(a_ens[b:e].view(np.uint64), a_alone.view(np.uint64)), f"system {s}"
