"""Ensemble (batching) inputs: many independent Plummer spheres of uneven size.

System s has N_s particles, N_s = floor(2**u), u uniform in [log2 nmin,
log2 nmax) from a seeded generator; its particles are a Plummer sphere
(plummer.h's algorithm, seed base_seed + s) scaled to total mass 1, virial
radius 1 like every single system.  The systems are concatenated in order,
the layout bonsai_set_systems expects.
"""
from __future__ import annotations

import numpy as np

from .treecode import plummer


def system_sizes(nsys: int, nmin: int = 1 << 10, nmax: int = 1 << 18, seed: int = 12345) -> np.ndarray:
    rng = np.random.default_rng(seed)
    u = rng.uniform(np.log2(nmin), np.log2(nmax), nsys)
    return np.floor(2.0 ** u).astype(np.int32)


def plummer_ensemble(counts, base_seed: int = 19810614):
    """(pos, vel) float32 (sum(counts), 4) arrays, system s from seed base_seed + s."""
    counts = np.asarray(counts, np.int64)
    n = int(counts.sum())
    pos = np.empty((n, 4), np.float32)
    vel = np.empty((n, 4), np.float32)
    off = 0
    for s, c in enumerate(counts):
        p, v = plummer(int(c), base_seed + s)
        pos[off:off + c] = p
        vel[off:off + c] = v
        off += int(c)
    return pos, vel
