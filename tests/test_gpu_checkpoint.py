"""Checkpoint / resume through Tipsy snapshots: a run stopped after two
steps, its velocities synchronised (bonsai_sync_velocities), written and read
back into a new handle, continues bit for bit like the uninterrupted run."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_checkpoint_resume_is_bit_exact(tmp_path):
    import bonsai2_b200 as B
    n = 65536
    p0, v0 = B.plummer(n, 7)
    prm = dict(eps=0.01, theta=0.5, dt=1.0 / 64)

    a = B.Treecode(**prm)
    a.alloc(n)
    a.h_ptclPos[:] = p0
    a.h_ptclVel[:] = v0
    a.ptcl_h2d()
    a.step(4, graph=True)
    assert a.synchronize() == 0
    a.ptcl_d2h()
    want_p, want_v = a.h_ptclPos.copy(), a.h_ptclVel.copy()
    a.close()

    b = B.Treecode(**prm)
    b.alloc(n)
    b.h_ptclPos[:] = p0
    b.h_ptclVel[:] = v0
    b.ptcl_h2d()
    b.step(2, graph=True)
    b.sync_velocities()
    assert b.synchronize() == 0
    b.ptcl_d2h()
    f = str(tmp_path / "ckpt.tipsy")
    B.write_tipsy(f, b.h_ptclPos, b.h_ptclVel, time=2 * prm["dt"])
    b.close()

    t, pos, vel, ids = B.read_tipsy(f)
    assert t == 2 * prm["dt"] and np.array_equal(ids, np.arange(n))
    c = B.Treecode(**prm)
    c.alloc(n)
    c.h_ptclPos[:] = pos
    c.h_ptclVel[:] = vel
    c.ptcl_h2d()
    c.step(2, graph=True)
    assert c.synchronize() == 0
    c.ptcl_d2h()
    assert np.array_equal(c.h_ptclPos.view(np.uint32), want_p.view(np.uint32))
    assert np.array_equal(c.h_ptclVel.view(np.uint32), want_v.view(np.uint32))
    c.close()
