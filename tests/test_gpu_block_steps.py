"""Block time steps (per-particle power-of-two steps, kick-drift-kick)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PRM = dict(eps=0.01, theta=0.5, dt=1.0 / 32)


def _load(t, p, v):
    t.alloc(p.shape[0])
    t.h_ptclPos[:] = p
    t.h_ptclVel[:] = v
    t.ptcl_h2d()


def test_single_level_is_the_plain_step():
    import bonsai2_b200 as B
    p, v = B.plummer(32768, 3)
    a = B.Treecode(**PRM)
    _load(a, p, v)
    a.step(4, graph=True)
    a.sync_velocities()  # the plain run's pending closing kick
    assert a.synchronize() == 0
    a.ptcl_d2h()
    b = B.Treecode(**PRM)
    _load(b, p, v)
    b.set_block_steps(0, 0.2)
    b.block_step(4)
    assert b.synchronize() == 0
    b.ptcl_d2h()
    assert np.array_equal(a.h_ptclPos.view(np.uint32), b.h_ptclPos.view(np.uint32))
    assert np.array_equal(a.h_ptclVel.view(np.uint32), b.h_ptclVel.view(np.uint32))
    assert np.all(b.levels() == 0)
    a.close()
    b.close()


def test_single_level_is_the_plain_step_in_double_single():
    import bonsai2_b200 as B
    p, v = B.galaxy(16384, seed=4)
    p[:, :3] += 1000.0
    out = []
    for block in (False, True):
        t = B.Treecode(**PRM)
        t.set_precision(1)
        t.set_particles_f64(p, v)
        if block:
            t.set_block_steps(0, 0.2)
            t.block_step(3)
        else:
            t.step(3, graph=True)
            t.sync_velocities()
        assert t.synchronize() == 0
        out.append(t.get_particles_f64())
        t.close()
    assert np.array_equal(out[0][0].view(np.uint64), out[1][0].view(np.uint64))
    assert np.array_equal(out[0][1].view(np.uint32), out[1][1].view(np.uint32))


def test_levels_follow_the_criterion_and_energy_is_kept():
    import bonsai2_b200 as B
    n, K, eta = 65536, 3, 0.05
    p, v = B.plummer(n, 11)
    t = B.Treecode(**PRM)
    _load(t, p, v)
    t.set_block_steps(K, eta)
    t.block_step(1)
    e0 = t.computeEnergies()
    t.block_step(4)
    assert t.synchronize() == 0
    e1 = t.computeEnergies()
    lev = t.levels()
    a = t.get_acc()
    # the criterion in float, in the kernel's operation order
    ax, ay, az = a[:, 0], a[:, 1], a[:, 2]
    am = np.sqrt((ax * ax + ay * ay) + az * az).astype(np.float32)
    dti = (np.float32(eta) * np.sqrt(np.float32(PRM["eps"]) / am)).astype(np.float32)
    dtk = np.ldexp(np.float32(PRM["dt"]), -lev.astype(np.int32)).astype(np.float32)
    assert lev.max() <= K
    assert np.all((dtk <= dti) | (lev == K))  # no particle steps longer than its criterion allows
    assert len(np.unique(lev)) >= 2           # the sphere's centre and halo take different steps
    # energy: relative change over four big steps
    assert abs(e1[3] - e0[3]) / abs(e0[3]) < 1e-4
    t.close()


def test_block_steps_accepted_for_ensembles_rejected_before_enabling():
    import bonsai2_b200 as B
    t = B.Treecode(**PRM)
    t.set_systems(np.array([100, 200], np.int32))
    assert t._L.bonsai_set_block_steps(t.handle, 2, 0.2) == 0
    assert t._L.bonsai_set_block_steps(t.handle, 2, 0.0) == -4  # eta must be > 0
    u = B.Treecode(**PRM)
    u.alloc(100)
    assert u._L.bonsai_block_step(u.handle, 1) == -3
    t.close()
    u.close()


def test_block_steps_in_an_ensemble_are_each_system_alone():
    """Block time steps inside an ensemble: every system's positions,
    velocities and levels after two big steps equal, bit for bit, those of the
    system stepped alone (a substep rebuilds the tree when any system has a
    particle ending a step there; the others only drift, as they do alone)."""
    import bonsai2_b200 as B
    from bonsai2_b200.ensemble import plummer_ensemble
    counts = np.array([3000, 7000, 2, 4500], np.int32)
    pos, vel = plummer_ensemble(counts, base_seed=41)
    prm = dict(PRM, dt=1.0 / 16)
    t = B.Treecode(**prm)
    t.set_systems(counts)
    t.h_ptclPos[:] = pos
    t.h_ptclVel[:] = vel
    t.ptcl_h2d()
    t.set_block_steps(2, 0.4)
    t.block_step(2)
    assert t.synchronize() == 0
    t.ptcl_d2h()
    lev = t.levels()
    es = t.system_energies()
    P, V = t.h_ptclPos.copy(), t.h_ptclVel.copy()
    t.close()
    assert len(np.unique(lev)) >= 2  # particles on different levels
    off = np.concatenate([[0], np.cumsum(counts)])
    for s in range(len(counts)):
        b, e = int(off[s]), int(off[s + 1])
        u = B.Treecode(**prm)
        _load(u, np.ascontiguousarray(pos[b:e]), np.ascontiguousarray(vel[b:e]))
        u.set_block_steps(2, 0.4)
        u.block_step(2)
        assert u.synchronize() == 0
        u.ptcl_d2h()
        assert np.array_equal(u.h_ptclPos.view(np.uint32), P[b:e].view(np.uint32)), f"positions of system {s}"
        assert np.array_equal(u.h_ptclVel.view(np.uint32), V[b:e].view(np.uint32)), f"velocities of system {s}"
        assert np.array_equal(u.levels(), lev[b:e]), f"levels of system {s}"
        np.testing.assert_allclose(u.computeEnergies(), es[s], rtol=1e-12, atol=1e-15)
        u.close()
