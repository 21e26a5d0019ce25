"""Ensemble (batching) inputs: many independent Plummer spheres of uneven size.

System s has N_s particles, N_s = floor(2**u), u uniform in [log2 nmin,
log2 nmax) from a seeded generator; its particles are a Plummer sphere
(plummer.h's algorithm, seed base_seed + s) scaled to total mass 1, virial
radius 1 like every single system.  The systems are concatenated in order,
the layout bonsai_set_systems expects.

Across GPUs the ensemble shards without any exchange: the systems are
partitioned over the ranks by estimated work (partition_systems), every rank
advances its own systems as an ensemble of its own (shard), and the only
communication is the final gather of per-system results to rank 0
(gather_systems).  A system's results do not depend on which other systems
share its ensemble, so the split gives every system exactly the result it gets
in one process.  The reference holds one tree per process and has no
multi-GPU path at all (read_tipsy.h:20,36 keep only a disabled procs/rank
stub).
"""
from __future__ import annotations

import numpy as np

from .treecode import plummer


def system_sizes(nsys: int, nmin: int = 1 << 10, nmax: int = 1 << 18, seed: int = 12345) -> np.ndarray:
    rng = np.random.default_rng(seed)
    u = rng.uniform(np.log2(nmin), np.log2(nmax), nsys)
    return np.floor(2.0 ** u).astype(np.int32)


def plummer_ensemble(counts, base_seed: int = 19810614, seeds=None):
    """(pos, vel) float32 (sum(counts), 4) arrays, system s from seed
    base_seed + s (or seeds[s]: a rank generating only its own systems passes
    their global seeds)."""
    counts = np.asarray(counts, np.int64)
    seeds = base_seed + np.arange(len(counts)) if seeds is None else np.asarray(seeds, np.int64)
    n = int(counts.sum())
    pos = np.empty((n, 4), np.float32)
    vel = np.empty((n, 4), np.float32)
    off = 0
    for c, sd in zip(counts, seeds):
        p, v = plummer(int(c), int(sd))
        pos[off:off + c] = p
        vel[off:off + c] = v
        off += int(c)
    return pos, vel


def system_work(counts) -> np.ndarray:
    """Estimated step cost of each system: N log2 N (tree depth times
    particles; the walk's interactions per particle grow with log N)."""
    c = np.asarray(counts, np.float64)
    return c * np.log2(np.maximum(c, 2.0))


def partition_systems(counts, world: int, work=None) -> list:
    """Systems of each rank (sorted index arrays): longest-processing-time
    first -- systems by decreasing work, each to the rank with the least work
    so far (ties: the lower rank), so every rank's total is within the
    largest system's work of the mean.  Deterministic: every rank computes the
    same partition from the same counts."""
    if world < 1:
        raise ValueError("world must be >= 1")
    w = system_work(counts) if work is None else np.asarray(work, np.float64)
    order = np.argsort(-w, kind="stable")
    load = np.zeros(world)
    owner = np.empty(len(w), np.int64)
    for s in order:
        r = int(np.argmin(load))
        owner[s] = r
        load[r] += w[s]
    return [np.flatnonzero(owner == r) for r in range(world)]


def shard(counts, pos, vel, systems):
    """This rank's ensemble: (counts, pos, vel) of the given systems, in
    ascending system order, concatenated as bonsai_set_systems expects."""
    counts = np.asarray(counts, np.int64)
    off = np.concatenate([[0], np.cumsum(counts)])
    systems = np.asarray(systems, np.int64)
    if systems.size == 0:
        return (np.zeros(0, np.int32), np.zeros((0, 4), pos.dtype), np.zeros((0, 4), vel.dtype))
    idx = np.concatenate([np.arange(off[s], off[s + 1]) for s in systems])
    return counts[systems].astype(np.int32), np.ascontiguousarray(pos[idx]), np.ascontiguousarray(vel[idx])


def gather_systems(dist, systems, per_system, nsys: int):
    """The final result gather: every rank passes its systems' rows
    (per_system[k] belongs to systems[k]); rank 0 gets the (nsys, ...) array
    in system order, the other ranks None.  dist is torch.distributed with an
    initialised process group, or None for one process."""
    per_system = np.asarray(per_system)
    if dist is None:
        parts = [(np.asarray(systems), per_system)]
    else:
        parts = [None] * dist.get_world_size()
        dist.all_gather_object(parts, (np.asarray(systems), per_system))
        if dist.get_rank() != 0:
            return None
    out = np.empty((nsys,) + per_system.shape[1:], per_system.dtype)
    seen = np.zeros(nsys, bool)
    for sy, rows in parts:
        if np.any(seen[sy]):
            raise RuntimeError("a system was returned by two ranks")
        seen[sy] = True
        out[sy] = rows
    if not seen.all():
        raise RuntimeError("systems missing from the gather")
    return out
