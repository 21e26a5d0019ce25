"""The allocation-free FP64 direct-sum checker (bonsai_direct_fp64_noalloc).

It exists for callers that cannot allocate device memory -- their GPU memory
is owned by another framework's allocator, or their loop must not pay
cudaMalloc's device-wide synchronisation -- so it takes device pointers and
keeps its scratch in a fixed 2 MiB array inside the library.  Checked here
through the C ABI against the existing entry point (bonsai_direct_fp64) on two
calls in a row, plus the size limit.  This file is collected last so that a
run stopping at the first failure has run every other test first; it also
passes alone in a fresh process (the first call does the per-device set-up).
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_matches_direct_fp64_twice(lib):
    import torch

    import bonsai2_b200 as B

    n, eps = 20000, 0.01
    pos, vel = B.plummer(n, 77)
    t = B.Treecode(eps=eps, theta=0.4)
    t.alloc(n)
    t.h_ptclPos[:] = pos
    t.h_ptclVel[:] = vel
    t.ptcl_h2d()
    d_pos = torch.from_numpy(pos).cuda()
    stream = torch.cuda.current_stream()
    eps2 = float(np.float32(eps)) ** 2
    rng = np.random.default_rng(5)
    for call, ns in enumerate((700, 1500)):
        sample = np.ascontiguousarray(rng.choice(n, ns, replace=False).astype(np.int32))
        d_sample = torch.from_numpy(sample).cuda()
        d_out = torch.full((ns, 4), float("nan"), dtype=torch.float64, device="cuda")
        rc = lib.bonsai_direct_fp64_noalloc(ctypes.c_void_p(d_pos.data_ptr()), n,
                                            ctypes.c_void_p(d_sample.data_ptr()), ns, eps2, 1,
                                            ctypes.c_void_p(d_out.data_ptr()), ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0, "call %d: %d" % (call, rc)
        stream.synchronize()
        got = d_out.cpu().numpy()
        ref = t.direct_fp64(sample, include_self=True)
        assert np.allclose(got, ref, rtol=1e-10, atol=1e-13), "call %d" % call
    t.close()


def test_noalloc_rejects_oversize(lib):
    import torch

    n = 100
    d_pos = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    ns = 65537
    d_sample = torch.zeros(ns, dtype=torch.int32, device="cuda")
    d_out = torch.zeros((ns, 4), dtype=torch.float64, device="cuda")
    rc = lib.bonsai_direct_fp64_noalloc(ctypes.c_void_p(d_pos.data_ptr()), n, ctypes.c_void_p(d_sample.data_ptr()),
                                        ns, 1e-4, 1, ctypes.c_void_p(d_out.data_ptr()), None)
    assert rc == -6
    assert b"65536" in lib.bonsai_error_string(rc)
