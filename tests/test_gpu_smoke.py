"""__graft_entry__.smoke(): the small end-to-end check (Plummer N = 4096: box,
keys, tree and groups bit-exact against the oracle, forces against the FP64
direct sum, one leapfrog step) runs clean on the GPU."""
import os
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_smoke():
    sys.path.insert(0, ROOT)
    import __graft_entry__ as g
    g.smoke()
