"""Tipsy snapshots on the host (no GPU): the library's writer and reader
against the reference's record layout (tipsydefs.h) and, where it was built
here, the reference's own reader (oracle/_ref/ref_tipsy_read, compiled from
read_tipsy.h by oracle/build_ref.sh)."""
import os
import struct
import subprocess

import numpy as np
import pytest

from bonsai2_b200 import read_tipsy, write_tipsy
from bonsai2_b200._lib import BonsaiError

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_READER = os.path.join(ROOT, "oracle", "_ref", "ref_tipsy_read")


def _particles(n, seed=0):
    rng = np.random.default_rng(seed)
    pos = rng.standard_normal((n, 4)).astype(np.float32)
    pos[:, 3] = rng.uniform(1e-6, 1e-3, n).astype(np.float32)
    vel = rng.standard_normal((n, 4)).astype(np.float32)
    vel[:, 3] = np.float32(0.01)
    ids = rng.permutation(n).astype(np.int32)
    return pos, vel, ids


def test_round_trip(tmp_path):
    pos, vel, ids = _particles(1000)
    f = str(tmp_path / "a.tipsy")
    write_tipsy(f, pos, vel, ids, time=1.25, ndark=600)
    t, p, v, i = read_tipsy(f)
    assert t == 1.25
    assert np.array_equal(p, pos) and np.array_equal(v, vel) and np.array_equal(i, ids)
    assert os.path.getsize(f) == 32 + 600 * 36 + 400 * 44


def test_reads_reference_layout(tmp_path):
    # a file packed by hand from tipsydefs.h: header, 2 dark then 1 star record
    f = str(tmp_path / "b.tipsy")
    with open(f, "wb") as fh:
        fh.write(struct.pack("=diiiii4x", 0.5, 3, 3, 0, 2, 1))
        fh.write(struct.pack("=8fi", 1.0, 2.0, 3.0, 4.0, 5.0, 6.0, 7.0, 0.1, 42))
        fh.write(struct.pack("=8fi", 1.5, 2.5, 3.5, 4.5, 5.5, 6.5, 7.5, 0.2, 43))
        fh.write(struct.pack("=10fi", 9.0, 1.0, 1.0, 1.0, 2.0, 2.0, 2.0, 0.7, 0.8, 0.3, 44))
    t, p, v, i = read_tipsy(f)
    assert t == 0.5
    assert np.array_equal(p, np.array([[2, 3, 4, 1], [2.5, 3.5, 4.5, 1.5], [1, 1, 1, 9]], np.float32))
    assert np.array_equal(v, np.array([[5, 6, 7, 0.1], [5.5, 6.5, 7.5, 0.2], [2, 2, 2, 0.3]], np.float32))
    assert list(i) == [42, 43, 44]


@pytest.mark.skipif(not os.path.exists(REF_READER), reason="reference Tipsy reader not built (oracle/build_ref.sh)")
def test_reference_reader_reads_our_snapshot(tmp_path):
    pos, vel, ids = _particles(777, seed=3)
    f = str(tmp_path / "c.tipsy")
    out = str(tmp_path / "c.bin")
    write_tipsy(f, pos, vel, ids, time=2.0, ndark=300)
    subprocess.run([REF_READER, f, out], check=True, capture_output=True)
    raw = open(out, "rb").read()
    n = struct.unpack("=i", raw[:4])[0]
    assert n == 777
    body = np.frombuffer(raw[4:], np.uint8)
    p = body[:n * 16].view(np.float32).reshape(n, 4)
    v = body[n * 16:n * 32].view(np.float32).reshape(n, 4)
    i = body[n * 32:n * 36].view(np.int32)
    assert np.array_equal(p, pos) and np.array_equal(v, vel) and np.array_equal(i, ids)


def test_errors(tmp_path):
    with pytest.raises(BonsaiError) as e:
        read_tipsy(str(tmp_path / "missing.tipsy"))
    assert e.value.code == -7
    pos, vel, ids = _particles(10)
    f = str(tmp_path / "d.tipsy")
    write_tipsy(f, pos, vel, ids)
    with open(f, "r+b") as fh:
        fh.truncate(32 + 5 * 36)
    with pytest.raises(BonsaiError) as e:
        read_tipsy(f)
    assert e.value.code == -7
