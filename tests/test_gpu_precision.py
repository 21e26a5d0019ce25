"""Double-single positions (precision form) on the GPU.

Accuracy is judged the reference's way, against the FP64 direct sum, here on
the exact (double) positions.  The composite galaxy is used at the origin and
moved to |x| ~ 1e4, where the float spacing (~1e-3) is comparable to the
bulge's particle separations: FP32 positions lose them there, double-single
positions must not."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

THETA = 0.4


def _forces(pos64, vel, precision, theta=THETA, eps=0.01, nleaf=16, ncrit=64, theta_mode=None):
    import bonsai2_b200 as B
    t = B.Treecode(eps=eps, theta=theta, ncrit=ncrit, nleaf=nleaf)
    t.set_precision(precision)
    t.set_particles_f64(pos64, vel)
    t.buildTree(nleaf)
    t.computeMultipoles()
    t.makeGroups(5, ncrit)
    if theta_mode is not None:
        ng = t.groups().shape[0]
        B.treecode._check(t._L.bonsai_set_theta_mode(t.handle, 2, 0.25, 1.25), "theta mode")
        th = np.full(ng, theta_mode, np.float32)
        B.treecode._check(t._L.bonsai_set_group_theta(t.handle, B.treecode._p(th), ng), "group theta")
    t.computeForces(False)
    assert t.synchronize() == 0
    acc = t.get_acc().astype(np.float64)
    return t, acc


def _reference(pos64, vel, sample, eps=0.01):
    import bonsai2_b200 as B
    t = B.Treecode(eps=eps, theta=THETA)
    t.set_precision(1)
    t.set_particles_f64(pos64, vel)
    ref = t.direct_fp64(sample, include_self=True)
    t.close()
    return ref


def _err(acc, ref, sample):
    return np.linalg.norm(acc[sample, :3] - ref[:, :3], axis=1) / np.linalg.norm(ref[:, :3], axis=1)


def test_split_round_trip():
    import bonsai2_b200 as B
    pos, vel = B.galaxy(4096, seed=3)
    pos[:, :3] += np.array([1000.0, -700.0, 500.0])
    t = B.Treecode()
    t.set_precision(1)
    t.set_particles_f64(pos, vel)
    p, v, _ = t.get_particles_f64()
    hi = pos[:, :3].astype(np.float32).astype(np.float64)
    lo = (pos[:, :3] - hi).astype(np.float32).astype(np.float64)
    assert np.array_equal(p[:, :3], hi + lo)
    assert np.abs(p[:, :3] - pos[:, :3]).max() < 1e-9
    t.close()


def test_galaxy_far_from_origin_keeps_accuracy():
    import bonsai2_b200 as B
    n = 1 << 16
    pos, vel = B.galaxy(n, seed=11)
    rng = np.random.default_rng(5)
    # half the samples in the bulge (the last 10 % of particles)
    sample = np.concatenate([rng.choice(int(0.9 * n), 256, replace=False),
                             int(0.9 * n) + rng.choice(n - int(0.9 * n), 256, replace=False)]).astype(np.int32)
    res = {}
    for label, shift in (("origin", 0.0), ("far", 1.0)):
        p = pos.copy()
        p[:, :3] += shift * np.array([1.0e4, -7.0e3, 5.0e3])
        ref = _reference(p, vel, sample)
        for prec in (0, 1):
            t, acc = _forces(p, vel, prec)
            res[(label, prec)] = _err(acc, ref, sample)
            t.close()
    med = {k: float(np.median(v)) for k, v in res.items()}
    p99 = {k: float(np.percentile(v, 99)) for k, v in res.items()}
    # at the origin both forms are multipole-limited and alike
    assert med[("origin", 1)] < 1e-3 and med[("origin", 0)] < 1e-3
    assert med[("origin", 1)] < 1.5 * med[("origin", 0)]
    # far away the double-single walk keeps its accuracy ...
    assert med[("far", 1)] < 1.5 * med[("origin", 1)]
    assert p99[("far", 1)] < 2.0 * p99[("origin", 1)]
    # ... and FP32 positions do not
    assert p99[("far", 0)] > 5.0 * p99[("far", 1)]


def test_per_group_theta_equal_to_fixed_is_exact_in_double_single():
    import bonsai2_b200 as B
    pos, vel = B.galaxy(1 << 15, seed=2)
    pos[:, :3] += 300.0
    t0, a0 = _forces(pos, vel, 1)
    t1, a1 = _forces(pos, vel, 1, theta_mode=THETA)
    assert np.array_equal(a0.view(np.uint64), a1.view(np.uint64))
    t0.close()
    t1.close()


def test_double_single_drift_keeps_small_steps():
    """Displacements far below the float spacing at |x| = 1000 accumulate in
    the low part; forces are negligible (tiny masses)."""
    import bonsai2_b200 as B
    n = 64
    rng = np.random.default_rng(0)
    pos = np.zeros((n, 4))
    pos[:, :3] = 1000.0 + rng.uniform(0, 50, (n, 3))
    pos[:, 3] = 1e-30
    vel = np.zeros((n, 4), np.float32)
    vel[:, 0] = 1e-6
    dt = 1.0 / 64
    out = {}
    for prec in (0, 1):
        t = B.Treecode(eps=0.01, theta=0.5, dt=dt)
        t.set_precision(prec)
        t.set_particles_f64(pos, vel)
        t.step(100, graph=True)
        assert t.synchronize() == 0
        out[prec] = t.get_particles_f64()[0]
        t.close()
    want = 100 * np.float64(np.float32(1e-6)) * dt
    moved1 = out[1][:, 0] - pos[:, 0]
    moved0 = out[0][:, 0] - pos[:, 0].astype(np.float32).astype(np.float64)
    np.testing.assert_allclose(moved1, want, rtol=1e-4)
    assert np.all(moved0 == 0.0)  # each step is below half an ulp of the float position


def test_precision_accepted_for_ensembles_and_reset_by_set_systems():
    """Double-single positions work inside ensembles (bit-identity per system:
    test_gpu_ensemble.py); a new ensemble layout starts in float positions."""
    import bonsai2_b200 as B
    t = B.Treecode()
    t.set_systems(np.array([100, 200], np.int32))
    assert t._L.bonsai_set_precision(t.handle, 1) == 0
    t.set_systems(np.array([50, 50, 200], np.int32))
    assert t._L.bonsai_set_precision(t.handle, 2) == -4  # modes are 0 and 1
    t.close()


def test_autotune_restores_double_single_state():
    import bonsai2_b200 as B
    pos, vel = B.galaxy(1 << 15, seed=8)
    pos[:, :3] += 1.0e4
    t = B.Treecode(eps=0.01, theta=0.5)
    t.set_precision(1)
    t.set_particles_f64(pos, vel)
    before = t.get_particles_f64()
    t.autotune(nleaf=(8, 16), ncrit=(32, 64), steps=1)
    after = t.get_particles_f64()
    assert np.array_equal(before[0].view(np.uint64), after[0].view(np.uint64))
    assert np.array_equal(before[1].view(np.uint32), after[1].view(np.uint32))
    t.close()
