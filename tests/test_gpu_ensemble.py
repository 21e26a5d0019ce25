"""Ensembles of independent systems (batching form): every system advanced in
the same launches must give, bit for bit, what the system gives alone.

The single-system path is itself pinned to the oracle (test_gpu_parity.py),
so bit-identity with it carries that parity over to every system of an
ensemble.  Edge systems of 1 and 2 particles are included."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PARAMS = dict(eps=0.01, theta=0.5, nleaf=16, ncrit=64, level_split=5, dt=1.0 / 64)


def _ensemble_inputs(counts, seed=777):
    from bonsai2_b200.ensemble import plummer_ensemble
    return plummer_ensemble(counts, base_seed=seed)


def _offsets(counts):
    return np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)


def _run(t, pos, vel, steps, eager):
    t.h_ptclPos[:] = pos
    t.h_ptclVel[:] = vel
    t.ptcl_h2d()
    stats = None
    if eager:
        for _ in range(steps):
            t.buildTree(t.nLeaf)
            t.computeMultipoles()
            t.makeGroups(5, t.nCrit)
            stats = t.computeForces(True)
            t.moveParticles()
    else:
        t.step(steps, graph=True)
    assert t.synchronize() == 0
    t.ptcl_d2h()
    return t.h_ptclPos.copy(), t.h_ptclVel.copy(), t.get_acc(), stats


def _alone(pos, vel, steps, eager, params=PARAMS, layout=0):
    import bonsai2_b200 as B
    t = B.Treecode(**params)
    t.set_walk_layout(layout)
    t.alloc(pos.shape[0])
    out = _run(t, pos, vel, steps, eager)
    e = t.computeEnergies()
    t.close()
    return out, e


@pytest.mark.parametrize("eager", [False, True])
def test_ensemble_bit_identical_to_alone(eager):
    import bonsai2_b200 as B
    from bonsai2_b200.ensemble import system_sizes
    counts = np.concatenate([[1, 2, 17], system_sizes(13, 1 << 8, 1 << 14, seed=5)]).astype(np.int32)
    pos, vel = _ensemble_inputs(counts)
    steps = 3
    t = B.Treecode(**PARAMS)
    t.set_systems(counts)
    p, v, a, stats = _run(t, pos, vel, steps, eager)
    es = t.system_energies()
    off = _offsets(counts)
    sum_app = sum_dir = 0
    for s in range(len(counts)):
        b, e = off[s], off[s + 1]
        (pa, va, aa, st), ea = _alone(pos[b:e], vel[b:e], steps, eager)
        assert np.array_equal(p[b:e].view(np.uint32), pa.view(np.uint32)), f"positions of system {s}"
        assert np.array_equal(v[b:e].view(np.uint32), va.view(np.uint32)), f"velocities of system {s}"
        assert np.array_equal(a[b:e].view(np.uint32), aa.view(np.uint32)), f"accelerations of system {s}"
        # FP64 sums in another grouping (chunks of the ensemble vs blocks alone): equal to
        # rounding; momentum terms are cancellations of O(1e-3) terms, hence the absolute floor
        np.testing.assert_allclose(es[s], ea, rtol=1e-12, atol=1e-15)
        if eager:
            sum_dir += st[0] * (e - b)
            sum_app += st[2] * (e - b)
    if eager:
        n = int(off[-1])
        # {<direct>, max direct, <approx>, max approx}: per-particle sums add up exactly
        assert round(stats[0] * n) == round(sum_dir)
        assert round(stats[2] * n) == round(sum_app)
    t.close()


def test_ensemble_direct_sum_is_per_system():
    import bonsai2_b200 as B
    counts = np.array([300, 1, 4000, 57], np.int32)
    pos, vel = _ensemble_inputs(counts, seed=31)
    t = B.Treecode(**PARAMS)
    t.set_systems(counts)
    t.h_ptclPos[:] = pos
    t.h_ptclVel[:] = vel
    t.ptcl_h2d()
    off = _offsets(counts)
    sample = np.array([0, 299, 300, 301, 2000, 4300, 4357], np.int32)
    d = t.direct_fp64(sample)
    for k, i in enumerate(sample):
        s = int(np.searchsorted(off, i, side="right") - 1)
        q = pos[off[s]:off[s + 1]].astype(np.float64)
        dr = q[:, :3] - pos[i, :3].astype(np.float64)
        r2 = (dr * dr).sum(1) + np.float64(np.float32(0.01)) ** 2
        rinv = 1.0 / np.sqrt(r2)
        ref = np.concatenate([(q[:, 3] * rinv ** 3)[:, None] * dr, -(q[:, 3] * rinv)[:, None]], 1).sum(0)
        np.testing.assert_allclose(d[k], ref, rtol=1e-10, atol=1e-12)
    t.close()


def test_ensemble_rejects_bad_counts():
    import bonsai2_b200 as B
    from bonsai2_b200._lib import BonsaiError
    t = B.Treecode(**PARAMS)
    with pytest.raises(BonsaiError):
        t.set_systems(np.array([10, 0, 5], np.int32))
    t.set_systems(np.array([10, 5], np.int32))
    assert t._L.bonsai_set_block_steps(t.handle, 2, 0.05) == 0  # block time steps inside an ensemble
    assert t._L.bonsai_set_block_steps(t.handle, 17, 0.05) != 0  # more levels than the 16 supported
    t.close()


def _ds_inputs(counts, seed=91):
    """float64 galaxies, each moved far from the origin by its own offset."""
    import bonsai2_b200 as B
    rng = np.random.default_rng(seed)
    ps, vs = [], []
    for s, c in enumerate(counts):
        p, v = B.galaxy(int(c), seed=seed + s)
        p[:, :3] += rng.uniform(-2.0e4, 2.0e4, 3)
        ps.append(p)
        vs.append(v)
    return np.concatenate(ps), np.concatenate(vs)


def _ds_run(t, pos, vel, steps, eager):
    t.set_precision(1)
    t.set_particles_f64(pos, vel)
    if eager:
        for _ in range(steps):
            t.buildTree(t.nLeaf)
            t.computeMultipoles()
            t.makeGroups(5, t.nCrit)
            t.computeForces(False)
            t.moveParticles()
    else:
        t.step(steps, graph=True)
    assert t.synchronize() == 0
    return t.get_particles_f64()


@pytest.mark.parametrize("eager", [False, True])
def test_ensemble_double_single_bit_identical_to_alone(eager):
    """Double-single positions inside an ensemble: systems far from the origin,
    each with its own offset, advance bit for bit as they do alone (positions
    hi + lo, velocities, accelerations), and the FP64 checker sums each sample
    over its own system's hi + lo positions."""
    import bonsai2_b200 as B
    counts = np.array([1, 2, 700, 5000, 3000], np.int32)
    pos, vel = _ds_inputs(counts)
    off = _offsets(counts)
    t = B.Treecode(**PARAMS)
    t.set_systems(counts)
    p, v, a = _ds_run(t, pos, vel, 3, eager)
    sample = np.array([0, 1, 2, 3, 500, 703, 4000, 8702], np.int32)
    d_ens = t.direct_fp64(sample, include_self=True)
    t.close()
    for s in range(counts.shape[0]):
        b, e = off[s], off[s + 1]
        u = B.Treecode(**PARAMS)
        u.alloc(int(e - b))
        pa, va, aa = _ds_run(u, pos[b:e], vel[b:e], 3, eager)
        inside = sample[(sample >= b) & (sample < e)]
        d_alone = u.direct_fp64((inside - b).astype(np.int32), include_self=True) if inside.size else None
        u.close()
        assert np.array_equal(p[b:e].view(np.uint64), pa.view(np.uint64)), f"positions of system {s}"
        assert np.array_equal(v[b:e].view(np.uint32), va.view(np.uint32)), f"velocities of system {s}"
        assert np.array_equal(a[b:e].view(np.uint32), aa.view(np.uint32)), f"accelerations of system {s}"
        if inside.size:
            k = np.searchsorted(sample, inside)
            np.testing.assert_allclose(d_ens[k], d_alone, rtol=1e-12, atol=1e-12)


def _forces(t, pos, vel, mode=0, theta_g=None, weights=None):
    """Eager force evaluation with fixed (0), network (1) or given (2) angles.
    The network's relative mode reads the previous evaluation's accelerations:
    the first evaluation after loading is its fixed-angle fallback, the second
    uses the network."""
    from bonsai2_b200 import learned
    t.h_ptclPos[:] = pos
    t.h_ptclVel[:] = vel
    t.ptcl_h2d()
    if mode == 1:
        learned.set_weights(t, weights)
    learned.set_theta_mode(t, mode)
    for _ in range(2 if mode == 1 else 1):
        t.buildTree(t.nLeaf)
        t.computeMultipoles()
        t.makeGroups(5, t.nCrit)
        if mode == 2:
            learned.set_group_theta(t, np.full(t.groups().shape[0], theta_g, np.float32))
        t.computeForces(True)
    assert t.synchronize() == 0
    return t.get_acc()


def test_ensemble_per_group_angles():
    """Per-group opening criteria inside an ensemble: every group at the fixed
    angle (mode 2) is the fixed-angle walk bit for bit, and the network's
    bounds (mode 1: features normalised per system, each group's scale from
    its system's previous accelerations) give each system, bit for bit, what
    it gets alone."""
    import bonsai2_b200 as B
    from bonsai2_b200 import learned
    counts = np.array([300, 1, 4000, 57, 9000, 2], np.int32)
    pos, vel = _ensemble_inputs(counts, seed=31)
    off = _offsets(counts)
    t = B.Treecode(**PARAMS)
    t.set_systems(counts)  # allocates for sum(counts)
    a_fixed = _forces(t, pos, vel, 0)
    a_const = _forces(t, pos, vel, 2, theta_g=PARAMS["theta"])
    assert np.array_equal(a_fixed.view(np.uint32), a_const.view(np.uint32))
    w = learned.init_weights(4)
    a_net = _forces(t, pos, vel, 1, weights=w)
    sc = learned.group_scale(t)
    # finite everywhere (systems of 1 and 2 particles have degenerate features
    # and no acceleration but the floor) and varying from group to group
    assert np.isfinite(sc).all() and (sc > 0).all() and sc.std() > 0
    assert not np.array_equal(a_net.view(np.uint32), a_fixed.view(np.uint32))
    t.close()
    for s in range(counts.shape[0]):
        b, e = off[s], off[s + 1]
        u = B.Treecode(**PARAMS)
        u.alloc(int(e - b))
        a_alone = _forces(u, pos[b:e], vel[b:e], 1, weights=w)
        u.close()
        assert np.array_equal(a_net[b:e].view(np.uint32), a_alone.view(np.uint32)), f"system {s}"


def test_autotune_restores_state_and_keeps_bit_identity():
    import bonsai2_b200 as B
    from bonsai2_b200.ensemble import system_sizes
    counts = system_sizes(24, 1 << 9, 1 << 14, seed=9)
    pos, vel = _ensemble_inputs(counts, seed=99)
    t = B.Treecode(**PARAMS)
    t.set_systems(counts)
    t.h_ptclPos[:] = pos
    t.h_ptclVel[:] = vel
    t.ptcl_h2d()
    r = t.autotune(nleaf=(8, 16), ncrit=(32, 64, 128), steps=1)
    ms = r["ms"]
    assert r["nleaf"] in (8, 16) and r["ncrit"] in (32, 64, 128) and r["layout"] in (0, 1)
    assert np.all(ms[1] > 0)                        # full-warp layout: every candidate ran
    assert np.all(ms[0][:, :2] > 0) and np.all(ms[0][:, 2] == -1)  # no half-warp layout above nCrit 64
    chosen = ms[r["layout"]]
    assert chosen[chosen > 0].min() == ms[ms > 0].min()  # the fastest candidate was kept
    # the state was restored: stepping now equals a fresh ensemble with the chosen parameters
    t.step(2, graph=True)
    assert t.synchronize() == 0
    t.ptcl_d2h()
    p1 = t.h_ptclPos.copy()
    prm = dict(PARAMS, nleaf=r["nleaf"], ncrit=r["ncrit"])
    u = B.Treecode(**prm)
    u.set_walk_layout(r["layout"])
    u.set_systems(counts)
    p2, _, _, _ = _run(u, pos, vel, 2, eager=False)
    assert np.array_equal(p1.view(np.uint32), p2.view(np.uint32))
    # and each system still matches itself alone under the chosen parameters
    off = _offsets(counts)
    for s in (0, len(counts) // 2, len(counts) - 1):
        b, e = off[s], off[s + 1]
        (pa, _, _, _), _ = _alone(pos[b:e], vel[b:e], 2, False, params=prm, layout=r["layout"])
        assert np.array_equal(p2[b:e].view(np.uint32), pa.view(np.uint32))
    t.close()
    u.close()


def test_ensemble_512_systems_spot_check():
    """The batching configuration's shape (512 systems, N_s log-uniform in
    [2^10, 2^18], theta 0.5, eps 0.01), 2 graph steps, three systems checked
    against themselves alone."""
    import bonsai2_b200 as B
    from bonsai2_b200.ensemble import system_sizes
    counts = system_sizes(512, 1 << 10, 1 << 18, seed=2024)
    pos, vel = _ensemble_inputs(counts, seed=1)
    t = B.Treecode(**PARAMS)
    t.set_systems(counts)
    p, v, a, _ = _run(t, pos, vel, 2, eager=False)
    assert np.isfinite(a).all()
    off = _offsets(counts)
    for s in (0, int(np.argmax(counts)), 511):
        b, e = off[s], off[s + 1]
        (pa, va, aa, _), _ = _alone(pos[b:e], vel[b:e], 2, False)
        assert np.array_equal(p[b:e].view(np.uint32), pa.view(np.uint32))
        assert np.array_equal(a[b:e].view(np.uint32), aa.view(np.uint32))
    t.close()


@pytest.mark.parametrize("world", [2, 3])
def test_split_ensemble_bit_identical_to_one_process(world):
    """The multi-GPU split of the batching form, its ranks run one after
    another on this GPU: each rank's shard (systems partitioned by work,
    generated by their global seeds) advanced as its own ensemble gives every
    system, bit for bit, its result in the one-process ensemble; the gathered
    per-system energies equal the one-process ones to FP64 rounding."""
    import bonsai2_b200 as B
    from bonsai2_b200.ensemble import gather_systems, partition_systems, plummer_ensemble, system_sizes
    counts = np.concatenate([[1, 2], system_sizes(22, 1 << 8, 1 << 14, seed=9)]).astype(np.int32)
    pos, vel = plummer_ensemble(counts, base_seed=31)
    steps = 3
    t = B.Treecode(**PARAMS)
    t.set_systems(counts)
    p, v, a, _ = _run(t, pos, vel, steps, eager=False)
    t.computeEnergies()
    es = t.system_energies()
    t.close()
    off = _offsets(counts)
    parts = partition_systems(counts, world)
    rows, owners = [], []
    for r in range(world):
        mine = parts[r]
        cr = counts[mine].astype(np.int32)
        pr, vr = plummer_ensemble(cr, seeds=31 + mine)
        u = B.Treecode(**PARAMS)
        u.set_systems(cr)
        pu, vu, au, _ = _run(u, pr, vr, steps, eager=False)
        u.computeEnergies()
        rows.append(u.system_energies())
        owners.append(mine)
        u.close()
        loff = _offsets(cr)
        for k, s in enumerate(mine):
            b, e = off[s], off[s + 1]
            lb, le = loff[k], loff[k + 1]
            assert np.array_equal(pu[lb:le].view(np.uint32), p[b:e].view(np.uint32)), f"positions of system {s}"
            assert np.array_equal(vu[lb:le].view(np.uint32), v[b:e].view(np.uint32)), f"velocities of system {s}"
            assert np.array_equal(au[lb:le].view(np.uint32), a[b:e].view(np.uint32)), f"accelerations of system {s}"
    E = gather_systems(None, np.concatenate(owners), np.concatenate(rows), len(counts))
    np.testing.assert_allclose(E, es, rtol=1e-12, atol=1e-15)
