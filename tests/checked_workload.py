"""Workloads run under the bounds-checked library (libbonsai_b200_checks.so,
loaded through BONSAI_B200_LIB by tests/test_gpu_checked.py in a child
process).  Each case exercises one family of kernels or one overflow path and
records the status the step returned and the bounds violations it caused;
the violation word is reset between cases.  Prints one JSON object.

Not a test module itself (no test_ prefix): the parent test asserts on the
output."""
import json
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import bonsai2_b200 as B  # noqa: E402
from bonsai2_b200 import learned  # noqa: E402
from bonsai2_b200.treecode import _check, _p  # noqa: E402


def _uniform(n, seed):
    rng = np.random.default_rng(seed)
    p = np.zeros((n, 4), np.float32)
    p[:, :3] = rng.uniform(-1, 1, (n, 3))
    p[:, 3] = 1.0 / n
    return p, np.zeros((n, 4), np.float32)


def _load(t, pos, vel):
    t.alloc(pos.shape[0])
    t.h_ptclPos[:] = pos
    t.h_ptclVel[:] = vel
    t.ptcl_h2d()


def _eager(t, nleaf, ncrit, level_split=5):
    t.buildTree(nleaf)
    t.computeMultipoles()
    t.makeGroups(level_split, ncrit)
    t.computeForces(True)
    t.moveParticles()
    t.computeEnergies()


def case_plummer():
    pos, vel = B.plummer(1 << 16)
    t = B.Treecode(eps=0.01, theta=0.5, dt=1.0 / 64)
    _load(t, pos, vel)
    _eager(t, 16, 64)
    st = [t.synchronize()]
    t.step(3, graph=True)
    st.append(t.synchronize())
    t.close()
    return st


def case_leaf_and_group_sizes():
    pos, vel = B.plummer(20000, 5)
    st = []
    for nleaf, ncrit, layout in ((1, 16, 0), (8, 32, 0), (64, 128, 0), (16, 64, 1), (24, 17, 0)):
        t = B.Treecode(eps=0.01, theta=0.6, nleaf=nleaf, ncrit=ncrit)
        t.set_walk_layout(layout)
        _load(t, pos, vel)
        _eager(t, nleaf, ncrit, 3)
        st.append(t.synchronize())
        t.close()
    return st


def case_ensemble():
    counts = np.array([1, 300, 4000, 57, 20000, 2], np.int32)
    rng = np.random.default_rng(3)
    parts = [B.plummer(int(c), int(rng.integers(1, 1 << 30))) for c in counts]
    pos = np.concatenate([p for p, _ in parts])
    vel = np.concatenate([v for _, v in parts])
    t = B.Treecode(eps=0.01, theta=0.5, dt=1.0 / 64)
    t.set_systems(counts)
    _load(t, pos, vel)
    t.step(2, graph=True)
    st = [t.synchronize()]
    t.direct_fp64(np.array([0, 1, 300, 4356, 24357], np.int32))
    st.append(t.synchronize())
    t.autotune(nleaf=(8, 16), ncrit=(32, 64), steps=1)
    st.append(t.synchronize())
    t.close()
    return st


def case_double_single():
    pos, vel = B.galaxy(1 << 15, seed=4)
    pos[:, :3] += 1.0e4
    t = B.Treecode(eps=0.01, theta=0.5, dt=1.0 / 64)
    t.set_precision(1)
    t.set_particles_f64(pos, vel)
    t.step(2, graph=True)
    st = [t.synchronize()]
    t.buildTree(16)
    t.computeMultipoles()
    t.makeGroups(5, 64)
    t.computeForces(False)
    t.compute_forces_fp64()
    st.append(t.synchronize())
    t.close()
    return st


def case_block_steps():
    pos, vel = B.plummer(1 << 15, 9)
    t = B.Treecode(eps=0.01, theta=0.5, dt=1.0 / 32)
    _load(t, pos, vel)
    t.set_block_steps(3, 0.05)
    t.block_step(2)
    st = [t.synchronize()]
    t.close()
    return st


def case_per_group_theta():
    pos, vel = B.plummer(1 << 15, 11)
    t = B.Treecode(eps=0.01, theta=0.5)
    _load(t, pos, vel)
    t.buildTree(16)
    t.computeMultipoles()
    t.makeGroups(5, 64)
    ng = t.groups().shape[0]
    learned.set_theta_mode(t, 2)
    learned.set_group_theta(t, np.random.default_rng(1).uniform(0.3, 1.0, ng).astype(np.float32))
    t.computeForces(True)
    st = [t.synchronize()]
    learned.set_weights(t, learned.init_weights(2))
    learned.set_theta_mode(t, 1)
    t.step(2, graph=True)
    st.append(t.synchronize())
    t.close()
    return st


def case_cell_capacity_overflow():
    # graphs captured for a uniform cube, replayed on pairs 1e-5 apart (nLeaf 1):
    # the cell arrays overflow, the build reports it and writes nothing past them
    pos, vel = _uniform(4096, 5)
    t = B.Treecode(eps=0.01, theta=0.5, nleaf=1)
    _load(t, pos, vel)
    t.step(1, graph=True)
    st = [t.synchronize()]
    b = pos.copy()
    b[1::2, :3] = b[0::2, :3] + np.float32(1e-5)
    t.h_ptclPos[:] = b
    t.ptcl_h2d()
    t.step(1, graph=True)
    st.append(t._L.bonsai_synchronize(t.handle))
    t.close()
    return st


def case_walk_list_overflow():
    pos, vel = _uniform(1 << 18, 4)
    t = B.Treecode(eps=0.01, theta=0.02)
    _load(t, pos, vel)
    t.buildTree(1)
    t.computeMultipoles()
    t.makeGroups(5, 64)
    t._L.bonsai_compute_forces(t.handle, 0, None)
    st = [t._L.bonsai_synchronize(t.handle)]
    t.close()
    return st


def case_coincident():
    pos, vel = B.plummer(4096, 2)
    pos[:100, :3] = pos[0, :3]
    t = B.Treecode(eps=0.01, theta=0.5)
    _load(t, pos, vel)
    t.buildTree(16)
    t.computeMultipoles()
    t.makeGroups(5, 64)
    t._L.bonsai_compute_forces(t.handle, 0, None)
    st = [t._L.bonsai_synchronize(t.handle)]
    t.close()
    return st


CASES = [case_plummer, case_leaf_and_group_sizes, case_ensemble, case_double_single, case_block_steps,
         case_per_group_theta, case_cell_capacity_overflow, case_walk_list_overflow, case_coincident]


def main():
    out = {"lib": os.environ.get("BONSAI_B200_LIB", ""), "selftest": B.load().bonsai_bounds_selftest(0)}
    b = B.bounds_check(reset=True)
    out["checked"] = b["checked"]
    for case in CASES:
        st = case()
        b = B.bounds_check(reset=True)
        out[case.__name__] = {"status": [int(s) for s in st], "violations": b["count"], "first_site": b["first_site"]}
    print(json.dumps(out))


if __name__ == "__main__":
    main()
