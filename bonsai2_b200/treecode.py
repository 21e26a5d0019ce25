"""Python mirror of the reference's Treecode<float> surface over the C ABI.

Reference: code/Treecode.h:123-223 and its driver code/treecode.cu:61-168.
Same member names, parameters and call order:

    tree = Treecode(eps, theta, ncrit)        # Treecode.h:164
    tree.alloc(n)                             # Treecode.h:175
    tree.h_ptclPos[:] = ...; tree.h_ptclVel[:] = ...   (float4 x,y,z,m)
    tree.ptcl_h2d()                           # Treecode.h:207
    tree.buildTree(nLeaf)                     # Treecode.h:216
    tree.computeMultipoles()                  # Treecode.h:217
    tree.makeGroups(levelSplit, nCrit)        # Treecode.h:218
    stats = tree.computeForces(INTCOUNT)      # Treecode.h:219 -> double4
    tree.moveParticles()                      # Treecode.h:220
    tree.computeEnergies()                    # Treecode.h:221

Where the reference aborts (CUDA_SAFE_CALL, assert), this raises BonsaiError.
All compute runs in libbonsai_b200.so on the GPU; nothing here computes.
"""
from __future__ import annotations

import ctypes
import warnings

import numpy as np

from ._lib import BonsaiError, bonsai_params, bonsai_tree_info, load

STATUS_DEPTH = 2


def _p(a: np.ndarray):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.c_void_p)


def _check(rc: int, where: str):
    if rc < 0 or (rc > 0 and rc != STATUS_DEPTH):
        raise BonsaiError(rc, where)
    if rc == STATUS_DEPTH:
        warnings.warn("%s: tree deeper than 21 levels, a fat leaf was kept" % where)
    return rc


def default_params() -> bonsai_params:
    p = bonsai_params()
    load().bonsai_default_params(ctypes.byref(p))
    return p


def bounds_check(reset: bool = False) -> dict:
    """Violations recorded by a bounds-checked build of the library (loaded
    through BONSAI_B200_LIB = _lib.CHECKED_LIB_PATH): {"checked", "count",
    "first_site"}; checked is False for the normal build."""
    count = ctypes.c_uint(0)
    site = ctypes.c_uint(0)
    rc = load().bonsai_bounds_check(ctypes.byref(count), ctypes.byref(site), 1 if reset else 0)
    if rc < 0:
        raise BonsaiError(rc, "bonsai_bounds_check")
    return {"checked": rc == 1, "count": int(count.value), "first_site": int(site.value)}


def plummer(n: int, seed: int = 19810614):
    """Plummer sphere (the reference's plummer.h algorithm), float4 pos/vel."""
    pos = np.empty((n, 4), np.float32)
    vel = np.empty((n, 4), np.float32)
    _check(load().bonsai_plummer(n, seed, _p(pos), _p(vel)), "bonsai_plummer")
    return pos, vel


def galaxy(n: int, seed: int = 1):
    """Composite galaxy (halo + disk + bulge), positions as (n, 4) float64
    (x, y, z, m), velocities (n, 4) float32 (bonsai_galaxy)."""
    pos = np.empty((n, 4), np.float64)
    vel = np.empty((n, 4), np.float32)
    _check(load().bonsai_galaxy(n, seed, _p(pos), _p(vel)), "bonsai_galaxy")
    return pos, vel


def clustered_field(n: int, seed: int = 1, nclusters: int = 64):
    """Plummer subclusters plus a uniform background, float32 (n, 4) arrays."""
    pos = np.empty((n, 4), np.float32)
    vel = np.empty((n, 4), np.float32)
    _check(load().bonsai_clustered_field(n, seed, nclusters, _p(pos), _p(vel)), "bonsai_clustered_field")
    return pos, vel


def read_tipsy(path: str):
    """(time, pos4 (n,4) float32 = x,y,z,mass, vel4 (n,4) float32 = vx,vy,vz,eps,
    ids (n,) int32) from a Tipsy snapshot (bonsai_read_tipsy)."""
    L = load()
    t = ctypes.c_double(0.0)
    n = ctypes.c_int(0)
    _check(L.bonsai_read_tipsy(path.encode(), ctypes.byref(t), ctypes.byref(n), None, None, None), "read_tipsy")
    pos = np.empty((n.value, 4), np.float32)
    vel = np.empty((n.value, 4), np.float32)
    ids = np.empty(n.value, np.int32)
    _check(L.bonsai_read_tipsy(path.encode(), ctypes.byref(t), ctypes.byref(n), _p(pos), _p(vel), _p(ids)),
           "read_tipsy")
    return t.value, pos, vel, ids


def write_tipsy(path: str, pos4, vel4, ids=None, time: float = 0.0, ndark: int = None):
    """Writes a Tipsy snapshot: the first ndark particles (default all) as dark
    records, the rest as star records (bonsai_write_tipsy)."""
    p = np.ascontiguousarray(pos4, np.float32)
    v = np.ascontiguousarray(vel4, np.float32)
    i = None if ids is None else np.ascontiguousarray(ids, np.int32)
    n = p.shape[0]
    _check(load().bonsai_write_tipsy(path.encode(), float(time), n, n if ndark is None else ndark, _p(p), _p(v),
                                     _p(i)), "write_tipsy")


class Treecode:
    def __init__(self, eps: float = 0.01, theta: float = 0.75, ncrit: int = 64, nleaf: int = 16,
                 level_split: int = 5, dt: float = 1.0 / 64, device: int = 0):
        self._L = load()
        p = default_params()
        p.eps, p.theta, p.ncrit, p.nleaf, p.level_split, p.dt, p.device = eps, theta, ncrit, nleaf, level_split, dt, device
        self._params = p
        h = ctypes.c_void_p()
        _check(self._L.bonsai_create(ctypes.byref(p), ctypes.byref(h)), "bonsai_create")
        self._h = h
        self.nPtcl = 0
        self.nCrit = ncrit
        self.nLeaf = nleaf
        self.grav_potential = 0.0
        self.h_ptclPos = None
        self.h_ptclVel = None

    # -- lifetime -------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            self._L.bonsai_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def handle(self):
        return self._h

    # -- reference fields ------------------------------------------------------
    @property
    def theta(self) -> float:
        return float(self._params.theta)

    @theta.setter
    def theta(self, v: float):
        self._params.theta = v
        _check(self._L.bonsai_set_params(self._h, ctypes.byref(self._params)), "bonsai_set_params")

    @property
    def eps2(self) -> float:
        e = np.float32(self._params.eps)
        return float(e * e)

    @property
    def dt(self) -> float:
        return float(self._params.dt)

    @dt.setter
    def dt(self, v: float):
        self._params.dt = v
        _check(self._L.bonsai_set_params(self._h, ctypes.byref(self._params)), "bonsai_set_params")

    def get_nPtcl(self) -> int:
        return self.nPtcl

    def get_nCrit(self) -> int:
        return self.nCrit

    def get_nLeaf(self) -> int:
        return self.nLeaf

    # -- buffers ---------------------------------------------------------------
    def alloc(self, n: int):
        _check(self._L.bonsai_alloc(self._h, n), "bonsai_alloc")
        self.nPtcl = n
        self.h_ptclPos = np.zeros((n, 4), np.float32)
        self.h_ptclVel = np.zeros((n, 4), np.float32)

    def set_systems(self, counts):
        """Ensemble layout: system s owns counts[s] consecutive particles of
        h_ptclPos/h_ptclVel (no counterpart in the reference, which holds one
        tree per process).  Allocates like alloc(sum(counts))."""
        c = np.ascontiguousarray(counts, np.int32)
        _check(self._L.bonsai_set_systems(self._h, _p(c), c.shape[0]), "bonsai_set_systems")
        n = int(c.sum())
        self.nPtcl = n
        self.nsys = int(c.shape[0])
        self.h_ptclPos = np.zeros((n, 4), np.float32)
        self.h_ptclVel = np.zeros((n, 4), np.float32)

    def system_energies(self) -> np.ndarray:
        """(nsys, 8) energies per system, columns as computeEnergies."""
        ns = getattr(self, "nsys", 1)
        e = np.empty((ns, 8), np.float64)
        _check(self._L.bonsai_get_system_energies(self._h, _p(e)), "bonsai_get_system_energies")
        return e

    def set_precision(self, mode: int):
        """1: double-single positions (hi + lo float pairs, group-relative
        walk coordinates); 0: float positions.  Set before loading particles."""
        _check(self._L.bonsai_set_precision(self._h, mode), "bonsai_set_precision")

    def set_particles_f64(self, pos4: np.ndarray, vel4: np.ndarray):
        """Loads (n, 4) float64 positions (x, y, z, m) and float32 velocities."""
        p = np.ascontiguousarray(pos4, np.float64)
        v = np.ascontiguousarray(vel4, np.float32)
        _check(self._L.bonsai_set_particles_f64(self._h, _p(p), _p(v), p.shape[0]), "bonsai_set_particles_f64")
        if p.shape[0] != self.nPtcl:
            self.nPtcl = p.shape[0]
            self.h_ptclPos = np.zeros((self.nPtcl, 4), np.float32)
            self.h_ptclVel = np.zeros((self.nPtcl, 4), np.float32)

    def get_particles_f64(self):
        """(positions float64 hi + lo, velocities, accelerations), caller order."""
        n = self.nPtcl
        p = np.empty((n, 4), np.float64)
        v = np.empty((n, 4), np.float32)
        a = np.empty((n, 4), np.float32)
        _check(self._L.bonsai_get_particles_f64(self._h, _p(p), _p(v), _p(a)), "bonsai_get_particles_f64")
        return p, v, a

    def compute_forces_fp64(self):
        """FP64 checker walk with the float walk's interaction lists:
        ((n, 4) float64 accelerations and potentials in caller order,
        interaction statistics as get_stats)."""
        a = np.empty((self.nPtcl, 4), np.float64)
        st = np.zeros(4, np.uint64)
        _check(self._L.bonsai_compute_forces_fp64(self._h, _p(a), _p(st)), "bonsai_compute_forces_fp64")
        return a, st

    def sync_velocities(self):
        """Forces at the current positions and the pending half kick applied,
        so that ptcl_d2h returns synchronised (x, v) for a checkpoint."""
        _check(self._L.bonsai_sync_velocities(self._h), "bonsai_sync_velocities")

    def set_block_steps(self, max_level: int, eta: float = 0.2):
        """Per-particle power-of-two time steps dt/2^k, k <= max_level
        (max_level < 0: off)."""
        _check(self._L.bonsai_set_block_steps(self._h, max_level, eta), "bonsai_set_block_steps")

    def block_step(self, nsteps: int = 1):
        _check(self._L.bonsai_block_step(self._h, nsteps), "bonsai_block_step")

    def levels(self) -> np.ndarray:
        out = np.empty(self.nPtcl, np.uint8)
        _check(self._L.bonsai_get_levels(self._h, _p(out)), "bonsai_get_levels")
        return out

    def set_walk_layout(self, layout: int):
        """0: two half-warps per group (nCrit <= 64), 1: one warp per group."""
        _check(self._L.bonsai_set_walk_layout(self._h, layout), "bonsai_set_walk_layout")

    def autotune(self, nleaf=(8, 16, 32), ncrit=(16, 32, 64, 128), steps: int = 2) -> dict:
        """Times every (layout, nLeaf, nCrit) candidate on the current
        particles (restored afterwards) and keeps the fastest."""
        nl = np.ascontiguousarray(nleaf, np.int32)
        nc = np.ascontiguousarray(ncrit, np.int32)
        res = np.empty((2, nl.shape[0], nc.shape[0]), np.float32)
        best = np.zeros(3, np.int32)
        _check(self._L.bonsai_autotune(self._h, _p(nl), nl.shape[0], _p(nc), nc.shape[0], steps, _p(res), _p(best)),
               "bonsai_autotune")
        self.nLeaf, self.nCrit = int(best[0]), int(best[1])
        self._params.nleaf, self._params.ncrit = self.nLeaf, self.nCrit
        return {"nleaf": int(best[0]), "ncrit": int(best[1]), "layout": int(best[2]), "ms": res}

    def ptcl_h2d(self):
        pos = np.ascontiguousarray(self.h_ptclPos, np.float32)
        vel = np.ascontiguousarray(self.h_ptclVel, np.float32)
        _check(self._L.bonsai_set_particles(self._h, _p(pos), _p(vel), pos.shape[0]), "bonsai_set_particles")

    def ptcl_d2h(self):
        """Copies positions and velocities back into h_ptclPos/h_ptclVel (caller order)."""
        _check(self._L.bonsai_get_particles(self._h, _p(self.h_ptclPos), _p(self.h_ptclVel), None),
               "bonsai_get_particles")

    def get_acc(self) -> np.ndarray:
        """Accelerations and potentials (ax, ay, az, phi) in caller order."""
        a = np.empty((self.nPtcl, 4), np.float32)
        _check(self._L.bonsai_get_particles(self._h, None, None, _p(a)), "bonsai_get_particles")
        return a

    # -- the step (Treecode.h:216-221) ------------------------------------------
    def buildTree(self, nLeaf: int = 16):
        self.nLeaf = nLeaf
        return _check(self._L.bonsai_build_tree(self._h, nLeaf), "buildTree")

    def computeMultipoles(self):
        return _check(self._L.bonsai_compute_multipoles(self._h), "computeMultipoles")

    def makeGroups(self, levelSplit: int = 1, nCrit: int = 64):
        self.nCrit = nCrit
        return _check(self._L.bonsai_make_groups(self._h, levelSplit, nCrit), "makeGroups")

    def computeForces(self, INTCOUNT: bool = True):
        """Returns (<direct>, max direct, <approx>, max approx) per particle when
        INTCOUNT, like the reference's double4; sets grav_potential."""
        out = np.zeros(4, np.float64)
        _check(self._L.bonsai_compute_forces(self._h, 1 if INTCOUNT else 0, _p(out)), "computeForces")
        if INTCOUNT:
            e = np.zeros(8, np.float64)
            _check(self._L.bonsai_compute_energies(self._h, _p(e)), "computeEnergies")
            self.grav_potential = float(e[1])
        return out

    def moveParticles(self):
        return _check(self._L.bonsai_move_particles(self._h), "moveParticles")

    def computeEnergies(self) -> np.ndarray:
        """(T, W, W_noself, T+W_noself, Px, Py, Pz, M) at the last force evaluation."""
        e = np.zeros(8, np.float64)
        _check(self._L.bonsai_compute_energies(self._h, _p(e)), "computeEnergies")
        return e

    def step(self, nsteps: int = 1, graph: bool = True):
        _check(self._L.bonsai_step(self._h, nsteps, 1 if graph else 0), "step")

    def synchronize(self) -> int:
        return _check(self._L.bonsai_synchronize(self._h), "synchronize")

    # -- inspection --------------------------------------------------------------
    def tree_info(self) -> dict:
        ti = bonsai_tree_info()
        _check(self._L.bonsai_get_tree_info(self._h, ctypes.byref(ti)), "get_tree_info")
        return {"ncells": ti.ncells, "nleaves": ti.nleaves, "nnodes": ti.nnodes, "nlevels": ti.nlevels,
                "ngroups": ti.ngroups, "status": ti.status, "level_beg": np.array(ti.level_beg[:], np.int32),
                "level_end": np.array(ti.level_end[:], np.int32)}

    def box(self) -> np.ndarray:
        b = np.empty(4, np.float32)
        _check(self._L.bonsai_get_box(self._h, _p(b)), "get_box")
        return b

    def keys(self) -> dict:
        n = self.nPtcl
        tk = np.empty(n, np.uint64)
        tp = np.empty(n, np.int32)
        pk = np.empty(n, np.uint64)
        pp = np.empty(n, np.int32)
        ids = np.empty(n, np.int32)
        _check(self._L.bonsai_get_keys(self._h, _p(tk), _p(tp), _p(pk), _p(pp), _p(ids)), "get_keys")
        return {"tree_keys": tk, "tree_perm": tp, "ph_keys": pk, "ph_perm": pp, "ids_at_build": ids}

    def cells(self, multipoles: bool = True) -> dict:
        ti = self.tree_info()
        C = ti["ncells"]
        cd = np.empty((C, 4), np.uint32)
        ll = np.empty(max(ti["nleaves"], 1), np.int32)
        par = np.empty(C, np.int32)
        out = {"cell_data": cd, "leaf_list": ll[:ti["nleaves"]], "parent": par, "info": ti}
        if multipoles:
            s = np.empty((C, 4), np.float32)
            m = np.empty((C, 4), np.float32)
            q0 = np.empty((C, 4), np.float32)
            q1 = np.empty((C, 2), np.float32)
            _check(self._L.bonsai_get_cells(self._h, _p(cd), _p(s), _p(m), _p(q0), _p(q1), _p(ll), _p(par)),
                   "get_cells")
            out.update(size=s, mono=m, quad0=q0, quad1=q1)
        else:
            _check(self._L.bonsai_get_cells(self._h, _p(cd), None, None, None, None, _p(ll), _p(par)), "get_cells")
        return out

    def groups(self) -> np.ndarray:
        G = self.tree_info()["ngroups"]
        g = np.empty((max(G, 1), 2), np.int32)
        _check(self._L.bonsai_get_groups(self._h, _p(g)), "get_groups")
        return g[:G]

    def walk_arrays(self) -> dict:
        n = self.nPtcl
        ip = np.empty((n, 4), np.float32)
        jp = np.empty((n, 4), np.float32)
        ac = np.empty((n, 4), np.float32)
        ids = np.empty(n, np.int32)
        _check(self._L.bonsai_get_walk_arrays(self._h, _p(ip), _p(jp), _p(ac), _p(ids)), "get_walk_arrays")
        return {"ipos": ip, "jpos": jp, "acc": ac, "ids": ids}

    def direct_fp64(self, sample, include_self: bool = True) -> np.ndarray:
        s = np.ascontiguousarray(sample, np.int32)
        out = np.empty((s.shape[0], 4), np.float64)
        _check(self._L.bonsai_direct_fp64(self._h, _p(s), s.shape[0], 1 if include_self else 0, _p(out)),
               "direct_fp64")
        return out
