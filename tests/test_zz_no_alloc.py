"""The allocation-free FP64 direct-sum checker (bonsai_direct_fp64_noalloc).

It exists for callers that cannot allocate device memory -- their GPU memory
is owned by another framework's allocator, or their loop must not pay
cudaMalloc's device-wide synchronisation -- so it takes device pointers and
keeps its scratch in a fixed 2 MiB array inside the library.  Checked here
through the C ABI against the CPU FP64 direct sum of the oracle on two calls
in a row, the larger first so that partial sums left in the shared array by
the first call would show in the second; plus an out-of-range sample index
(a NaN row, the other rows intact), the argument checks and the size limit.
This file is collected last so that a run stopping at the first failure has
run every other test first; it also passes alone in a fresh process (every
call looks the array up on the current device).
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _call(lib, d_pos, n, d_sample, ns, eps2, include_self, d_out, stream):
    return lib.bonsai_direct_fp64_noalloc(ctypes.c_void_p(d_pos.data_ptr()), n,
                                          ctypes.c_void_p(d_sample.data_ptr()), ns, eps2, include_self,
                                          ctypes.c_void_p(d_out.data_ptr()),
                                          ctypes.c_void_p(stream.cuda_stream) if stream is not None else None)


def test_noalloc_matches_oracle_twice(lib, oracle):
    import torch

    import bonsai2_b200 as B

    n, eps = 6000, 0.01
    pos, _ = B.plummer(n, 77)
    d_pos = torch.from_numpy(pos).cuda()
    stream = torch.cuda.current_stream()
    eps2 = float(np.float32(eps)) ** 2
    rng = np.random.default_rng(5)
    for call, (ns, self_term) in enumerate(((3000, 1), (400, 0))):
        sample = np.ascontiguousarray(rng.choice(n, ns, replace=False).astype(np.int32))
        d_sample = torch.from_numpy(sample).cuda()
        d_out = torch.full((ns, 4), float("nan"), dtype=torch.float64, device="cuda")
        rc = _call(lib, d_pos, n, d_sample, ns, eps2, self_term, d_out, stream)
        assert rc == 0, "call %d: %d" % (call, rc)
        stream.synchronize()
        got = d_out.cpu().numpy()
        ref = oracle.direct_fp64(pos, sample, eps, include_self=bool(self_term))
        assert np.allclose(got, ref, rtol=1e-10, atol=1e-13), "call %d: max diff %g" % (
            call, np.abs(got - ref).max())


def test_noalloc_out_of_range_index_gives_nan_row(lib, oracle):
    import torch

    import bonsai2_b200 as B

    n, eps = 3000, 0.01
    pos, _ = B.plummer(n, 78)
    d_pos = torch.from_numpy(pos).cuda()
    stream = torch.cuda.current_stream()
    sample = np.array([5, n, 17, -1, n - 1], np.int32)
    d_sample = torch.from_numpy(sample).cuda()
    d_out = torch.zeros((len(sample), 4), dtype=torch.float64, device="cuda")
    rc = _call(lib, d_pos, n, d_sample, len(sample), float(np.float32(eps)) ** 2, 1, d_out, stream)
    assert rc == 0
    stream.synchronize()
    got = d_out.cpu().numpy()
    bad = (sample < 0) | (sample >= n)
    assert np.isnan(got[bad]).all()
    ref = oracle.direct_fp64(pos, sample[~bad], eps, include_self=True)
    assert np.allclose(got[~bad], ref, rtol=1e-10, atol=1e-13)


def test_noalloc_rejects_bad_arguments_and_oversize(lib):
    import torch

    n = 100
    d_pos = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    ns = 65537
    d_sample = torch.zeros(ns, dtype=torch.int32, device="cuda")
    d_out = torch.zeros((ns, 4), dtype=torch.float64, device="cuda")
    rc = _call(lib, d_pos, n, d_sample, ns, 1e-4, 1, d_out, None)
    assert rc == -6
    assert b"65536" in lib.bonsai_error_string(rc)
    # eps2 = 0 with the i == j term summed would be 0/0: refused
    assert _call(lib, d_pos, n, d_sample, 10, 0.0, 1, d_out, None) == -4
    assert _call(lib, d_pos, n, d_sample, 10, -1.0, 0, d_out, None) == -4
