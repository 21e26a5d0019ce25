"""bonsai2_b200 -- B200-native (sm_100a) tree code: the per-step hot path of
Bonsai2 (PH keys + sort, octree, quadrupole multipoles, groups, warp tree
walk, leapfrog + energies) as hand-written CUDA behind a C ABI
(include/bonsai_b200.h), with a Python mirror of the reference's Treecode
class.  All compute is in libbonsai_b200.so; there is no CPU fallback."""
from ._lib import BonsaiError, load  # noqa: F401
from .treecode import (Treecode, bounds_check, clustered_field, default_params, galaxy, plummer, read_tipsy,  # noqa: F401
                       write_tipsy)

__all__ = ["Treecode", "plummer", "galaxy", "clustered_field", "read_tipsy", "write_tipsy", "default_params",
           "bounds_check", "BonsaiError", "load"]
