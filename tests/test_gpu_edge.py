"""GPU edge cases and size-independent properties at the full size.

Edge cases the reference's own debug checks cover (every particle in one leaf,
sum of group sizes = N, permutation consistency, PSHFL_SANITY_CHECK) and those
it cannot handle (N=1, coincident particles deeper than 21 levels, NaN input:
the reference traps or loops there; here they return a status code)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def full_tree(oracle, pos, vel, nleaf, ncrit, ls=5, theta=0.4, eps=0.01):
    import bonsai2_b200 as B
    t = B.Treecode(eps=eps, theta=theta, ncrit=ncrit, nleaf=nleaf, level_split=ls)
    t.alloc(pos.shape[0])
    t.h_ptclPos[:] = pos
    t.h_ptclVel[:] = vel
    t.ptcl_h2d()
    t.buildTree(nleaf)
    t.computeMultipoles()
    t.makeGroups(ls, ncrit)
    stats = t.computeForces(True)
    return t, stats


def check_against_oracle(oracle, t, pos, nleaf, ncrit, ls):
    box, _ = oracle.bbox(pos)
    assert np.array_equal(t.box(), box)
    T = oracle.OracleTree(pos, box, nleaf)
    c = t.cells(multipoles=False)
    assert c["info"]["ncells"] == T.ncells
    assert np.array_equal(c["cell_data"], T.cell_data())
    k = t.keys()
    leaf = T.nchild == 0
    for ci in np.nonzero(leaf)[0]:
        b, e = T.pbeg[ci], T.pend[ci]
        assert np.array_equal(np.sort(k["tree_perm"][b:e]), np.sort(T.perm[b:e]))
    pk = oracle.ph_keys(pos, box)
    pp = oracle.argsort_u64(pk)
    assert np.array_equal(k["ph_perm"], pp)
    gb, gn = oracle.make_groups(pk[pp], ls, ncrit)
    g = t.groups()
    assert np.array_equal(g[:, 0], gb) and np.array_equal(g[:, 1], gn)
    return T


@pytest.mark.parametrize("n", [1, 2, 3, 16, 17, 100, 4097])
def test_small_n(oracle, lib, n):
    p, v = oracle.plummer_float4(max(n, 64), 5)
    p, v = np.ascontiguousarray(p[:n]), np.ascontiguousarray(v[:n])
    t, stats = full_tree(oracle, p, v, 16, 64)
    check_against_oracle(oracle, t, p, 16, 64, 5)
    acc = t.get_acc().astype(np.float64)
    d = oracle.direct_fp64(p, np.arange(n), 0.01, include_self=True)
    err = np.linalg.norm(acc[:, :3] - d[:, :3], axis=1) / np.maximum(np.linalg.norm(d[:, :3], axis=1), 1e-30)
    if n > 1:
        assert np.median(err) < 1e-3
    else:
        assert np.all(acc[:, :3] == 0) and abs(acc[0, 3] + p[0, 3] / 0.01) < 1e-6 * abs(acc[0, 3])
    assert t.synchronize() == 0


@pytest.mark.parametrize("nleaf,ncrit", [(16, 32), (24, 64), (32, 64), (48, 128), (64, 64), (1, 16), (8, 100)])
def test_leaf_and_group_sizes(oracle, lib, nleaf, ncrit):
    p, v = oracle.plummer_float4(30000, 11)
    t, stats = full_tree(oracle, p, v, nleaf, ncrit)
    check_against_oracle(oracle, t, p, nleaf, ncrit, 5)
    acc = t.get_acc().astype(np.float64)
    samp = np.arange(0, 30000, 97)
    d = oracle.direct_fp64(p, samp, 0.01)
    err = np.linalg.norm(acc[samp, :3] - d[:, :3], axis=1) / np.linalg.norm(d[:, :3], axis=1)
    assert np.median(err) < 1e-3


@pytest.mark.parametrize("ls", [1, 3, 7])
def test_level_split(oracle, lib, ls):
    p, v = oracle.plummer_float4(20000, 3)
    t, _ = full_tree(oracle, p, v, 16, 64, ls=ls)
    check_against_oracle(oracle, t, p, 16, 64, ls)


def test_coincident_particles_depth_status(oracle, lib):
    # 40 particles at one point force the partition below level 21: the
    # reference recurses without bound; here a fat leaf is kept and flagged
    p, v = oracle.plummer_float4(5000, 2)
    p[100:140, :3] = p[7, :3]
    t, _ = full_tree(oracle, p, v, 16, 64)
    T = check_against_oracle(oracle, t, p, 16, 64, 5)
    assert T.overflow
    assert t.tree_info()["status"] & 2
    acc = t.get_acc()
    assert np.all(np.isfinite(acc))
    with pytest.warns(UserWarning):
        assert t.synchronize() == 2


def test_nonfinite_input_reports_status(oracle, lib):
    import bonsai2_b200 as B
    p, v = oracle.plummer_float4(4096, 2)
    p[10, 0] = np.nan
    t = B.Treecode(eps=0.01, theta=0.4)
    t.alloc(p.shape[0])
    t.h_ptclPos[:] = p
    t.h_ptclVel[:] = v
    t.ptcl_h2d()
    with pytest.raises(B.BonsaiError) as ei:
        t.buildTree(16)
        t.synchronize()
    assert ei.value.code & 8


def test_stage_order_errors(oracle, lib):
    import bonsai2_b200 as B
    p, v = oracle.plummer_float4(1000, 2)
    t = B.Treecode()
    t.alloc(1000)
    t.h_ptclPos[:] = p
    t.h_ptclVel[:] = v
    t.ptcl_h2d()
    with pytest.raises(B.BonsaiError):
        t.computeMultipoles()
    with pytest.raises(B.BonsaiError):
        t.computeForces()
    with pytest.raises(B.BonsaiError):
        t.moveParticles()


def test_energy_drift_short_run(oracle, lib):
    import bonsai2_b200 as B
    p, v = oracle.plummer_float4(65536)
    t = B.Treecode(eps=0.01, theta=0.4, dt=1.0 / 128)
    t.alloc(p.shape[0])
    t.h_ptclPos[:] = p
    t.h_ptclVel[:] = v
    t.ptcl_h2d()
    E = []
    for s in range(8):
        t.step(1, graph=True)
        E.append(t.computeEnergies()[3])
    assert t.synchronize() == 0
    E = np.array(E)
    assert abs(E[-1] - E[0]) / abs(E[0]) < 1e-4
    assert abs(t.computeEnergies()[7] - 1.0) < 1e-6


@pytest.mark.parametrize("precision", [0, 1])
def test_leapfrog_time_reversible(precision):
    """Kick-drift-kick with deterministic forces is time-reversible: K steps,
    synchronised velocities reversed, K steps back, and the particles return
    to their start up to rounding (amplified by the dynamics), for float and
    double-single positions.  Checks the merged kicks, the pending closing
    kick and its synchronisation together."""
    import bonsai2_b200 as B
    p, v = B.plummer(4096, 5)
    p64 = p.astype(np.float64)
    t = B.Treecode(eps=0.01, theta=0.5, dt=1.0 / 128)
    t.set_precision(precision)
    t.set_particles_f64(p64, v)
    K = 32
    t.step(K, graph=True)
    t.sync_velocities()
    x1, v1, _ = t.get_particles_f64()
    t.set_particles_f64(x1, -v1)
    t.step(K, graph=True)
    t.sync_velocities()
    x2, v2, _ = t.get_particles_f64()
    assert t.synchronize() == 0
    t.close()
    moved = np.linalg.norm(x1[:, :3] - p64[:, :3], axis=1)
    back = np.linalg.norm(x2[:, :3] - p64[:, :3], axis=1)
    assert np.median(moved) > 1e-2
    assert np.median(back) < 1e-3 * np.median(moved)
    assert np.percentile(back, 99) < 1e-2 * np.median(moved)
    dv = np.linalg.norm(v2[:, :3].astype(np.float64) + v[:, :3], axis=1)
    assert np.median(dv) < 1e-3 * np.median(np.linalg.norm(v[:, :3], axis=1))


def test_full_size_properties(lib):
    # the large benchmark configuration: N = 2^24 Plummer, theta 0.4, eps 0.005
    import bonsai2_b200 as B
    n = 1 << 24
    pos, vel = B.plummer(n, 19810614)
    t, stats = full_tree(None, pos, vel, 16, 64, eps=0.005)
    assert t.synchronize() == 0
    k = t.keys()
    assert np.all(k["tree_keys"][1:] >= k["tree_keys"][:-1])
    assert np.all(k["ph_keys"][1:] >= k["ph_keys"][:-1])
    assert np.array_equal(np.sort(k["tree_perm"]), np.arange(n))
    assert np.array_equal(np.sort(k["ph_perm"]), np.arange(n))
    c = t.cells(multipoles=False)
    cd = c["cell_data"]
    leaf = cd[:, 1] == 0xFFFFFFFF
    assert (cd[leaf, 3].astype(np.int64) - cd[leaf, 2]).sum() == n
    assert np.all(cd[leaf, 3] - cd[leaf, 2] <= 16)
    g = t.groups()
    assert g[:, 1].sum() == n and np.all(g[:, 1] <= 64)
    acc = t.get_acc().astype(np.float64)
    rng = np.random.default_rng(11)
    samp = rng.choice(n, 256, replace=False)
    d = t.direct_fp64(samp, include_self=True)
    err = np.linalg.norm(acc[samp, :3] - d[:, :3], axis=1) / np.linalg.norm(d[:, :3], axis=1)
    assert np.median(err) < 1e-3


def test_max_size_2p27_invariants():
    """N = 2^27 (134M particles, 8x the bench size, ~35 GB on the device): a
    Plummer profile drawn by inverse transform (fast on the host); sorted keys,
    permutations, leaf and group coverage, a graph step with no status, and the
    force error on a sample, so that no index or size overflows 32 bits on the
    way to the largest systems one B200 holds comfortably."""
    import bonsai2_b200 as B
    n = 1 << 27
    rng = np.random.default_rng(27)
    u = rng.uniform(1e-6, 0.99, n)
    r = 1.0 / np.sqrt(u ** (-2.0 / 3.0) - 1.0)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    pos = np.empty((n, 4), np.float32)
    pos[:, :3] = d * r[:, None]
    pos[:, 3] = 1.0 / n
    del u, r, d
    vel = np.zeros((n, 4), np.float32)
    t = B.Treecode(eps=0.005, theta=0.6, dt=1.0 / 128)
    t.alloc(n)
    t.h_ptclPos[:] = pos
    t.h_ptclVel[:] = vel
    t.ptcl_h2d()
    t.buildTree(16)
    t.computeMultipoles()
    t.makeGroups(5, 64)
    t.computeForces(False)
    assert t.synchronize() == 0
    k = t.keys()
    assert np.all(k["tree_keys"][1:] >= k["tree_keys"][:-1])
    assert np.all(k["ph_keys"][1:] >= k["ph_keys"][:-1])
    for perm in (k["tree_perm"], k["ph_perm"]):
        c = np.bincount(perm, minlength=n)
        assert c.shape[0] == n and c.min() == 1 and c.max() == 1
    del k
    cd = t.cells(multipoles=False)["cell_data"]
    leaf = cd[:, 1] == 0xFFFFFFFF
    assert (cd[leaf, 3].astype(np.int64) - cd[leaf, 2]).sum() == n
    del cd, leaf
    g = t.groups()
    assert g[:, 1].astype(np.int64).sum() == n and np.all(g[:, 1] <= 64)
    acc = t.get_acc().astype(np.float64)
    samp = np.random.default_rng(11).choice(n, 128, replace=False).astype(np.int32)
    ref = t.direct_fp64(samp, include_self=True)
    err = np.linalg.norm(acc[samp, :3] - ref[:, :3], axis=1) / np.linalg.norm(ref[:, :3], axis=1)
    assert np.median(err) < 1e-3
    t.step(1, graph=True)
    assert t.synchronize() == 0
    t.close()


def test_bounded_wait_reports_and_device_stays_usable():
    """A radix-sort pass whose first tile never starts: the next tile's
    look-back waits on a flag nothing sets, ends at its bound and reports
    BONSAI_STATUS_SORT_TIMEOUT; the device then runs a normal step."""
    import bonsai2_b200 as B
    L = B.load()
    r = L.bonsai_selftest_wait_bound(0)
    assert r >= 0 and (r & 64)
    p, v = B.plummer(4096, 3)
    t = B.Treecode(eps=0.01, theta=0.5)
    t.alloc(4096)
    t.h_ptclPos[:] = p
    t.h_ptclVel[:] = v
    t.ptcl_h2d()
    t.step(1, graph=True)
    assert t.synchronize() == 0
    assert np.isfinite(t.get_acc()).all()
    t.close()


def test_walk_level_list_overflow_reports_status():
    """A uniform cube at a tiny opening angle: breadth-first levels wider than
    a warp's list capacity.  The walk reports BONSAI_STATUS_WALK_STACK and
    marks the affected groups' forces NaN instead of writing past its lists."""
    import bonsai2_b200 as B
    n = 1 << 18
    rng = np.random.default_rng(4)
    p = np.zeros((n, 4), np.float32)
    p[:, :3] = rng.uniform(-1, 1, (n, 3))
    p[:, 3] = 1.0 / n
    v = np.zeros((n, 4), np.float32)
    t = B.Treecode(eps=0.01, theta=0.02)
    t.alloc(n)
    t.h_ptclPos[:] = p
    t.h_ptclVel[:] = v
    t.ptcl_h2d()
    t.buildTree(1)
    t.computeMultipoles()
    t.makeGroups(5, 64)
    assert t._L.bonsai_compute_forces(t.handle, 0, None) == 0  # the launch itself is fine
    assert t._L.bonsai_last_error(t.handle) & 4                # peek: the status stays set
    assert t._L.bonsai_last_error(t.handle) & 4
    with pytest.raises(B.BonsaiError) as e:
        B.treecode._check(t._L.bonsai_synchronize(t.handle), "walk")  # reported and cleared
    assert e.value.code & 4
    assert t._L.bonsai_last_error(t.handle) == 0
    a = t.get_acc()
    assert np.isnan(a[:, 0]).any()
    t.close()


def test_cell_capacity_overflow_in_graph_replay_then_recovery():
    """Graphs are captured with cell arrays sized for the particles of the
    time (plus a margin).  Particles that need many more cells (tightly bound
    pairs at nLeaf 1) overflow them on replay: the step reports
    BONSAI_STATUS_CELL_CAPACITY without writing past the arrays; an eager build
    regrows them and the next step is clean."""
    import bonsai2_b200 as B
    n = 4096
    rng = np.random.default_rng(5)
    a = np.zeros((n, 4), np.float32)
    a[:, :3] = rng.uniform(-1, 1, (n, 3))
    a[:, 3] = 1.0 / n
    v = np.zeros((n, 4), np.float32)
    t = B.Treecode(eps=0.01, theta=0.5, nleaf=1)
    t.alloc(n)
    t.h_ptclPos[:] = a
    t.h_ptclVel[:] = v
    t.ptcl_h2d()
    t.step(1, graph=True)
    assert t.synchronize() == 0
    cells_a = t.tree_info()["ncells"]
    b = a.copy()
    b[1::2, :3] = b[0::2, :3] + np.float32(1e-5)  # pairs 1e-5 apart: ~17 more levels each
    t.h_ptclPos[:] = b
    t.ptcl_h2d()
    t.step(1, graph=True)
    st = t._L.bonsai_synchronize(t.handle)
    assert st > 0 and (st & 1)
    t.buildTree(1)  # eager build: grows the cell arrays (and drops the graphs)
    assert t.tree_info()["ncells"] > 2 * cells_a
    t.h_ptclPos[:] = b
    t.ptcl_h2d()
    t.step(1, graph=True)
    assert t.synchronize() == 0
    assert np.isfinite(t.get_acc()).all()
    t.close()
