"""ctypes wrapper around oracle/bonsai_oracle.c -- the CPU restatement of the
Bonsai2 hot path.

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and by
bench.py's cpu_baseline / reference leg.  The product (bonsai2_b200) never
imports it.  See the header of bonsai_oracle.c for which reference lines each
function restates and how each one is pinned.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD_DIR = os.path.join(HERE, "_build")
LIB_PATH = os.path.join(BUILD_DIR, "liboracle.so")
SRC = os.path.join(HERE, "bonsai_oracle.c")

MAXL = 21


def build(force: bool = False) -> str:
    """Compile the C restatement into oracle/_build/liboracle.so."""
    os.makedirs(BUILD_DIR, exist_ok=True)
    if (not force and os.path.exists(LIB_PATH)
            and os.path.getmtime(LIB_PATH) >= os.path.getmtime(SRC)):
        return LIB_PATH
    tmp = LIB_PATH + ".tmp%d" % os.getpid()
    cmd = ["gcc", "-O2", "-fopenmp", "-fPIC", "-shared", "-std=gnu11", SRC, "-o", tmp, "-lm"]
    subprocess.check_call(cmd)
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.c_void_p
        i32, u32, f32, f64, i64 = ctypes.c_int, ctypes.c_uint, ctypes.c_float, ctypes.c_double, ctypes.c_long
        L.oracle_plummer.argtypes = [i64, u32, P, P, P]
        L.oracle_bbox.argtypes = [i32, P, P]
        L.oracle_bbox.restype = i32
        L.oracle_tree_keys.argtypes = [i32, P, P, P]
        L.oracle_ph_keys.argtypes = [i32, P, P, P]
        L.oracle_argsort_u64.argtypes = [i32, P, P]
        L.oracle_build_tree.argtypes = [i32, P, P, i32, i32, P, P, P, P, P, P, P, P, P, P]
        L.oracle_build_tree.restype = i32
        L.oracle_multipoles_ref.argtypes = [i32, P, P, P, f32, P, P, P, P]
        L.oracle_multipoles_fp64.argtypes = [i32, P, P, P, P]
        L.oracle_make_groups.argtypes = [i32, P, i32, i32, P, P]
        L.oracle_make_groups.restype = i32
        L.oracle_walk.argtypes = [i32, P, P, P, P, P, P, P, P, P, i32, i32, P, f32, P, P, P]
        L.oracle_walk.restype = i32
        L.oracle_direct_fp64.argtypes = [i32, P, i32, P, f64, i32, P]
        L.oracle_move.argtypes = [i32, P, P, P, f32, i32, f32, P]
        L.oracle_num_threads.restype = i32
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.c_void_p)


# ----------------------------------------------------------------------------
# thin numpy-facing helpers
# ----------------------------------------------------------------------------

def plummer(n: int, seed: int = 19810614):
    """Plummer sphere, restating code/plummer.h:9-138 (FP64, glibc rand)."""
    m = np.empty(n, np.float64)
    p = np.empty((n, 3), np.float64)
    v = np.empty((n, 3), np.float64)
    lib().oracle_plummer(n, seed, _p(m), _p(p), _p(v))
    return m, p, v


def plummer_float4(n: int, seed: int = 19810614):
    """Plummer converted to the reference's float4 layout (treecode.cu:65-87):
    pos=(x,y,z,m), vel=(vx,vy,vz,m)."""
    m, p, v = plummer(n, seed)
    pos = np.empty((n, 4), np.float32)
    vel = np.empty((n, 4), np.float32)
    pos[:, :3] = p
    pos[:, 3] = m
    vel[:, :3] = v
    vel[:, 3] = m
    return pos, vel


def bbox(pos4: np.ndarray):
    box = np.empty(4, np.float32)
    bad = lib().oracle_bbox(pos4.shape[0], _p(pos4), _p(box))
    return box, bad


def tree_keys(pos4, box):
    k = np.empty(pos4.shape[0], np.uint64)
    lib().oracle_tree_keys(pos4.shape[0], _p(pos4), _p(box), _p(k))
    return k


def ph_keys(pos4, box):
    k = np.empty(pos4.shape[0], np.uint64)
    lib().oracle_ph_keys(pos4.shape[0], _p(pos4), _p(box), _p(k))
    return k


def argsort_u64(keys):
    keys = np.ascontiguousarray(keys, np.uint64)
    perm = np.empty(keys.shape[0], np.int32)
    lib().oracle_argsort_u64(keys.shape[0], _p(keys), _p(perm))
    return perm


class OracleTree:
    """Canonical octree: cells level by level, key order inside a level."""

    def __init__(self, pos4, box, nleaf):
        n = pos4.shape[0]
        cap = max(2 * n + 64, 64)
        self.perm = np.empty(n, np.int32)
        arrs = [np.empty(cap, np.int32) for _ in range(6)]
        self.level_beg = np.zeros(32, np.int32)
        self.level_end = np.zeros(32, np.int32)
        ov = np.zeros(1, np.int32)
        nc = lib().oracle_build_tree(n, _p(pos4), _p(box), nleaf, cap, _p(self.perm),
                                     *[_p(a) for a in arrs], _p(self.level_beg), _p(self.level_end), _p(ov))
        if nc < 0:
            raise RuntimeError("oracle tree: cell capacity exceeded")
        self.ncells = nc
        self.level, self.pbeg, self.pend, self.first, self.nchild, self.parent = [a[:nc].copy() for a in arrs]
        self.overflow = bool(ov[0])
        self.nlevels = int(np.max(self.level)) if nc else 0

    def cell_data(self):
        """Reference CellData packing (Treecode.h:45-89) as uint32[C,4]."""
        c = np.empty((self.ncells, 4), np.uint32)
        par = np.where(self.parent < 0, 0, self.parent).astype(np.uint32)
        c[:, 0] = par | (self.level.astype(np.uint32) << np.uint32(27))
        leaf = self.nchild == 0
        y = (self.first.astype(np.int64) & 0x1FFFFFFF) | ((self.nchild.astype(np.int64) - 1) << 29)
        c[:, 1] = np.where(leaf, 0xFFFFFFFF, y & 0xFFFFFFFF).astype(np.uint32)
        c[:, 2] = self.pbeg
        c[:, 3] = self.pend
        return c


def multipoles_ref(pbeg, pend, jpos4, theta):
    nc = pbeg.shape[0]
    size4 = np.empty((nc, 4), np.float32)
    mono4 = np.empty((nc, 4), np.float32)
    q0 = np.empty((nc, 4), np.float32)
    q1 = np.empty((nc, 2), np.float32)
    pb = np.ascontiguousarray(pbeg, np.int32)
    pe = np.ascontiguousarray(pend, np.int32)
    lib().oracle_multipoles_ref(nc, _p(pb), _p(pe), _p(jpos4), np.float32(1.0 / theta),
                                _p(size4), _p(mono4), _p(q0), _p(q1))
    return size4, mono4, q0, q1


def multipoles_fp64(pbeg, pend, jpos4):
    nc = pbeg.shape[0]
    out = np.empty((nc, 16), np.float64)
    pb = np.ascontiguousarray(pbeg, np.int32)
    pe = np.ascontiguousarray(pend, np.int32)
    lib().oracle_multipoles_fp64(nc, _p(pb), _p(pe), _p(jpos4), _p(out))
    return out


def make_groups(sorted_keys, level_split, ncrit):
    n = sorted_keys.shape[0]
    gb = np.empty(max(n, 1), np.int32)
    gn = np.empty(max(n, 1), np.int32)
    sk = np.ascontiguousarray(sorted_keys, np.uint64)
    g = lib().oracle_make_groups(n, _p(sk), level_split, ncrit, _p(gb), _p(gn))
    return gb[:g].copy(), gn[:g].copy()


def walk(gbeg, gnp, ipos4, cell_data, cell_size4, mono4, quad0, quad1, l1_beg, l1_end, jpos4, eps,
         gsel=None):
    n = ipos4.shape[0]
    G = gbeg.shape[0]
    acc = np.zeros((n, 4), np.float32)
    na = np.zeros(G, np.int64)
    nd = np.zeros(G, np.int64)
    gb = np.ascontiguousarray(gbeg, np.int32)
    gn = np.ascontiguousarray(gnp, np.int32)
    if gsel is None:
        nsel, psel = G, None
    else:
        gsel = np.ascontiguousarray(gsel, np.int32)
        nsel, psel = gsel.shape[0], _p(gsel)
    err = lib().oracle_walk(nsel, psel, _p(gb), _p(gn), _p(ipos4), _p(np.ascontiguousarray(cell_data, np.uint32)),
                            _p(np.ascontiguousarray(cell_size4, np.float32)),
                            _p(np.ascontiguousarray(mono4, np.float32)),
                            _p(np.ascontiguousarray(quad0, np.float32)),
                            _p(np.ascontiguousarray(quad1, np.float32)),
                            l1_beg, l1_end, _p(jpos4), np.float32(np.float32(eps) * np.float32(eps)),
                            _p(acc), _p(na), _p(nd))
    if err:
        raise RuntimeError("oracle walk: list buffer overflow")
    return acc, na, nd


def direct_fp64(pos4, sample, eps, include_self=True):
    sample = np.ascontiguousarray(sample, np.int32)
    out = np.empty((sample.shape[0], 4), np.float64)
    e = float(np.float32(eps))
    lib().oracle_direct_fp64(pos4.shape[0], _p(pos4), sample.shape[0], _p(sample), e * e,
                             1 if include_self else 0, _p(out))
    return out


def move(pos4, vel4, acc4, dt, closing, eps):
    e = np.empty(8, np.float64)
    lib().oracle_move(pos4.shape[0], _p(pos4), _p(vel4), _p(acc4), np.float32(dt), 1 if closing else 0,
                      np.float32(eps), _p(e))
    return e


def num_threads() -> int:
    return int(lib().oracle_num_threads())


# ----------------------------------------------------------------------------
# composed reference step (used by the CPU baseline and the parity tests)
# ----------------------------------------------------------------------------

class OracleStep:
    """One force evaluation of the reference algorithm on the CPU.

    Order of operations and data flow (the reference's, treecode.cu:137-165):
    box -> keys -> tree (canonical) -> multipoles -> PH keys/sort -> groups ->
    walk.  Tie-breaks in both sorts are by input position, matching the CUDA
    path (the reference's own tie order is atomicAdd order).
    """

    def __init__(self, pos4, theta, eps, nleaf=16, ncrit=64, level_split=5):
        self.pos4 = np.ascontiguousarray(pos4, np.float32)
        self.theta, self.eps, self.nleaf, self.ncrit, self.level_split = theta, eps, nleaf, ncrit, level_split

    def build(self):
        p = self.pos4
        self.box, self.bad = bbox(p)
        self.tree = OracleTree(p, self.box, self.nleaf)
        self.jpos = p[self.tree.perm]
        return self

    def multipoles(self):
        t = self.tree
        self.size4, self.mono4, self.quad0, self.quad1 = multipoles_ref(t.pbeg, t.pend, self.jpos, self.theta)
        return self

    def groups(self):
        k = ph_keys(self.pos4, self.box)
        self.ph_perm = argsort_u64(k)
        self.ph_sorted = k[self.ph_perm]
        self.gbeg, self.gnp = make_groups(self.ph_sorted, self.level_split, self.ncrit)
        self.ipos = self.pos4[self.ph_perm]
        return self

    def forces(self, gsel=None):
        t = self.tree
        self.acc, self.napprox, self.ndirect = walk(
            self.gbeg, self.gnp, self.ipos, t.cell_data(), self.size4, self.mono4, self.quad0, self.quad1,
            int(t.level_beg[1]), int(t.level_end[1]), self.jpos, self.eps, gsel=gsel)
        return self
