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


def test_block_steps_rejected_for_ensembles_and_before_enabling():
    import bonsai2_b200 as B
    t = B.Treecode(**PRM)
    t.set_systems(np.array([100, 200], np.int32))
    assert t._L.bonsai_set_block_steps(t.handle, 2, 0.2) == -4
    u = B.Treecode(**PRM)
    u.alloc(100)
    assert u._L.bonsai_block_step(u.handle, 1) == -3
    t.close()
    u.close()
