"""Asynchronous host copies: the pipelined set / step / get sequence must give
bit for bit what the synchronous calls give, with downloads still in flight
while later steps run."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _pinned(L, n):
    ptr = L.bonsai_host_alloc(n * 16)
    assert ptr
    return ptr, np.ctypeslib.as_array((ctypes.c_float * (4 * n)).from_address(ptr)).reshape(n, 4)


def test_async_pipeline_matches_synchronous():
    import bonsai2_b200 as B
    from bonsai2_b200.treecode import _p
    L = B.load()
    n = 50000
    p0, v0 = B.plummer(n, 5)
    inputs = []
    for k in range(4):  # four different inputs, one per step
        p = p0.copy()
        p[:, 0] += 0.01 * k
        inputs.append((p, v0.copy()))
    # synchronous reference
    ref = []
    t = B.Treecode(eps=0.01, theta=0.5)
    t.alloc(n)
    for p, v in inputs:
        assert L.bonsai_set_particles(t.handle, _p(p), _p(v), n) == 0
        t.step(1, graph=True)
        a = np.empty((n, 4), np.float32)
        q = np.empty((n, 4), np.float32)
        assert L.bonsai_get_particles(t.handle, _p(q), None, _p(a)) == 0
        ref.append((q, a))
    assert t.synchronize() == 0
    t.close()
    # pipelined: pinned buffers, nothing waited for until the end
    u = B.Treecode(eps=0.01, theta=0.5)
    u.alloc(n)
    keep = []
    pins = []
    for p, v in inputs:
        pp, pa = _pinned(L, n)
        vp, va = _pinned(L, n)
        pa[:] = p
        va[:] = v
        qp, qa = _pinned(L, n)
        ap, aa = _pinned(L, n)
        pins += [pp, vp, qp, ap]
        assert L.bonsai_set_particles_async(u.handle, ctypes.c_void_p(pp), ctypes.c_void_p(vp), n) == 0
        u.step(1, graph=True)
        assert L.bonsai_get_particles_async(u.handle, ctypes.c_void_p(qp), None, ctypes.c_void_p(ap)) == 0
        keep.append((qa, aa))
    assert u.synchronize() == 0
    for (q, a), (qa, aa) in zip(ref, keep):
        assert np.array_equal(q.view(np.uint32), qa.view(np.uint32))
        assert np.array_equal(a.view(np.uint32), aa.view(np.uint32))
    u.close()
    for ptr in pins:
        L.bonsai_host_free(ptr)


def test_async_rejects_size_change():
    import bonsai2_b200 as B
    from bonsai2_b200.treecode import _p
    L = B.load()
    t = B.Treecode()
    p, v = B.plummer(1000, 1)
    assert L.bonsai_set_particles_async(t.handle, _p(p), _p(v), 1000) == -2  # not allocated
    t.alloc(1000)
    assert L.bonsai_set_particles_async(t.handle, _p(p[:500].copy()), _p(v[:500].copy()), 500) == -4
    t.close()
