"""Learned per-group opening angles: training-set generation, training and
use of the 16 -> 64 -> 64 -> 1 network of csrc/learned.cu.

Training pairs come from the plain method and the FP64 direct sum, both on
the GPU: for a random subset of groups and a few particles in each, the walk
runs with every group at each angle of a grid (theta mode 2) and the largest
angle whose error (geometric mean over the group's sampled particles of
|da|/|a| against the direct sum) stays below the target is the label.  The
network is trained with the library's own forward/backward kernels
(bonsai_mlp_train, Adam, full batch) and used in theta mode 1, where a
feature kernel and an FP16-weight inference kernel set each group's angle
inside the step.
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import BonsaiError, load
from .treecode import Treecode, _check, _p

NFEAT = 16
NWEIGHTS = 5313
LO, HI, OVER = 0.25, 1.25, 3.0


def init_weights(seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    H, F = 64, NFEAT
    parts = [rng.normal(0, np.sqrt(1.0 / F), H * F), np.zeros(H), rng.normal(0, np.sqrt(1.0 / H), H * H), np.zeros(H),
             rng.normal(0, np.sqrt(1.0 / H), H), [0.0]]
    return np.ascontiguousarray(np.concatenate(parts).astype(np.float32))


def loss_grad(X, y, w, lo=LO, hi=HI, over=OVER, device=0):
    X = np.ascontiguousarray(X, np.float32)
    y = np.ascontiguousarray(y, np.float32)
    w = np.ascontiguousarray(w, np.float32)
    g = np.empty(NWEIGHTS, np.float32)
    loss = ctypes.c_double(0)
    _check(load().bonsai_mlp_loss_grad(device, _p(X), _p(y), X.shape[0], _p(w), lo, hi, over, _p(g),
                                       ctypes.byref(loss)), "mlp_loss_grad")
    return loss.value, g


def train(X, y, w0=None, epochs=2000, lr=3e-3, lo=LO, hi=HI, over=OVER, device=0, seed=0):
    X = np.ascontiguousarray(X, np.float32)
    y = np.ascontiguousarray(y, np.float32)
    w = np.ascontiguousarray(init_weights(seed) if w0 is None else w0, np.float32).copy()
    loss = ctypes.c_double(0)
    _check(load().bonsai_mlp_train(device, _p(X), _p(y), X.shape[0], _p(w), epochs, lr, lo, hi, over,
                                   ctypes.byref(loss)), "mlp_train")
    return w, loss.value


def predict(X, w, lo=LO, hi=HI, device=0):
    X = np.ascontiguousarray(X, np.float32)
    w = np.ascontiguousarray(w, np.float32)
    out = np.empty(X.shape[0], np.float32)
    _check(load().bonsai_mlp_predict(device, _p(X), X.shape[0], _p(w), lo, hi, _p(out)), "mlp_predict")
    return out


def group_features(t: Treecode) -> np.ndarray:
    G = t.tree_info()["ngroups"]
    F = np.empty((max(G, 1), NFEAT), np.float32)
    ng = ctypes.c_int(0)
    _check(t._L.bonsai_get_group_features(t.handle, _p(F), ctypes.byref(ng)), "get_group_features")
    return F[:ng.value]


def set_group_theta(t: Treecode, theta):
    th = np.ascontiguousarray(theta, np.float32)
    _check(t._L.bonsai_set_group_theta(t.handle, _p(th), th.shape[0]), "set_group_theta")


def set_theta_mode(t: Treecode, mode: int, lo=LO, hi=HI):
    _check(t._L.bonsai_set_theta_mode(t.handle, mode, lo, hi), "set_theta_mode")


def set_weights(t: Treecode, w):
    w = np.ascontiguousarray(w, np.float32)
    _check(t._L.bonsai_set_mlp_weights(t.handle, _p(w), w.shape[0]), "set_mlp_weights")


def group_theta(t: Treecode) -> np.ndarray:
    G = t.tree_info()["ngroups"]
    out = np.empty(max(G, 1), np.float32)
    _check(t._L.bonsai_get_group_theta(t.handle, _p(out)), "get_group_theta")
    return out[:G]


DEFAULT_GRID = tuple(np.round(np.arange(0.30, 1.2501, 0.05), 2))


def group_interactions(t: Treecode) -> np.ndarray:
    """(G, 2) approximate and direct interaction counts per group of the last
    walk with per-group angles."""
    G = t.tree_info()["ngroups"]
    out = np.empty((max(G, 1), 2), np.uint32)
    _check(t._L.bonsai_get_group_interactions(t.handle, _p(out)), "get_group_interactions")
    return out[:G]


def training_tables(pos, vel, eps, thetas=DEFAULT_GRID, samples_per_group=8, max_groups=8192, seed=0, nleaf=16,
                    ncrit=64, level_split=5, device=0):
    """For a random subset of groups: features F (g, 16); error table E (g, k)
    = geometric mean over the group's sampled particles of |da|/|a| against
    the FP64 direct sum with every group at angle thetas[k]; cost table C
    (g, k) = 64 n_approx + 20 n_direct of the group's warp (the walk's model
    flops; a warp evaluates all its particle slots); group sizes (g,)."""
    n = pos.shape[0]
    t = Treecode(eps=eps, theta=0.5, ncrit=ncrit, nleaf=nleaf, level_split=level_split, device=device)
    try:
        t.alloc(n)
        t.h_ptclPos[:] = pos
        t.h_ptclVel[:] = vel
        t.ptcl_h2d()
        t.buildTree(nleaf)
        t.computeMultipoles()
        t.makeGroups(level_split, ncrit)
        F = group_features(t)
        groups = t.groups()
        G = groups.shape[0]
        ids = t.walk_arrays()["ids"]
        rng = np.random.default_rng(seed)
        gsel = np.sort(rng.choice(G, min(max_groups, G), replace=False))
        spos = []  # PH positions of the sampled particles
        owner = []
        for k, g in enumerate(gsel):
            pb, np_ = groups[g]
            take = rng.choice(np_, min(samples_per_group, np_), replace=False)
            spos.extend(pb + take)
            owner.extend([k] * len(take))
        spos = np.asarray(spos, np.int64)
        owner = np.asarray(owner, np.int64)
        ref = t.direct_fp64(ids[spos].astype(np.int32), include_self=True)
        refn = np.linalg.norm(ref[:, :3], axis=1)
        set_theta_mode(t, 2)
        E = np.zeros((gsel.shape[0], len(thetas)))
        C = np.zeros((gsel.shape[0], len(thetas)))
        for j, th in enumerate(thetas):
            set_group_theta(t, np.full(G, th, np.float32))
            t.computeForces(False)
            acc = t.walk_arrays()["acc"][spos].astype(np.float64)
            err = np.linalg.norm(acc[:, :3] - ref[:, :3], axis=1) / refn
            le = np.log(np.maximum(err, 1e-30))
            E[:, j] = np.exp(np.bincount(owner, weights=le, minlength=gsel.shape[0]) /
                             np.bincount(owner, minlength=gsel.shape[0]))
            cnt = group_interactions(t)[gsel].astype(np.float64)
            C[:, j] = 64.0 * cnt[:, 0] + 20.0 * cnt[:, 1]
        return F[gsel], E, C, groups[gsel, 1].astype(np.float64)
    finally:
        t.close()


def crossing_labels(E, thetas, target):
    """Per group, the angle at which its error crosses the target
    (interpolated linearly in log error between grid angles, clipped to the
    grid's ends): every group made equally accurate."""
    th = np.asarray(thetas, np.float64)
    lt = np.log(target)
    logE = np.log(np.maximum(E, 1e-30))
    label = np.full(E.shape[0], th[0])
    for g in range(E.shape[0]):
        above = np.nonzero(logE[g] > lt)[0]
        if above.size == 0:
            label[g] = th[-1]
            continue
        j = above[0]
        if j == 0:
            label[g] = th[0]
            continue
        e0, e1 = logE[g, j - 1], logE[g, j]
        f = (lt - e0) / (e1 - e0) if e1 > e0 else 0.0
        label[g] = th[j - 1] + f * (th[j] - th[j - 1])
    return label.astype(np.float32)


def _wmedian(x, w):
    o = np.argsort(x)
    cw = np.cumsum(w[o])
    return float(x[o][np.searchsorted(cw, 0.5 * cw[-1])])


def allocation_labels(E, C, sizes, thetas, target, fraction=0.9):
    """Per-group angles that minimise total walk cost for a given error
    budget: group g takes argmin_k C[g,k]/mean(C) + lam * log E[g,k] (a
    Lagrangian relaxation; groups whose error grows slowly with the angle get
    larger angles), lam bisected so that the particle-weighted geometric mean
    of the groups' errors is fraction * target.  (The budget is the geometric
    mean, not the median: a median budget is met by the easier half of the
    groups alone, and its optimum leaves the other half arbitrarily wrong.)
    Returns (labels, info); info compares the allocation's cost with the fixed
    angle of equal median on the same groups: the bound a per-group angle
    model can reach there."""
    th = np.asarray(thetas, np.float64)
    logE = np.log(np.maximum(E, 1e-30))
    Cn = C / C.mean()
    wts = sizes / sizes.sum()
    goal = np.log(fraction * target)
    rows = np.arange(E.shape[0])

    def alloc(lam):
        j = np.argmin(Cn + lam * logE, axis=1)
        return j, float((wts * logE[rows, j]).sum())

    lo, hi = 1e-4, 1e3
    for _ in range(60):
        mid = np.sqrt(lo * hi)
        if alloc(mid)[1] > goal:
            lo = mid
        else:
            hi = mid
    j, _ = alloc(hi)
    med = _wmedian(E[rows, j], sizes)
    cost = float(C[rows, j].sum())
    fixed_med = np.array([_wmedian(E[:, k], sizes) for k in range(len(th))])
    fixed_cost = C.sum(axis=0)
    # fixed angle cost at the allocation's median, log-log between grid angles
    fc = None
    o = np.argsort(fixed_med)
    fm, fcs = fixed_med[o], fixed_cost[o]
    for a in range(len(fm) - 1):
        if fm[a] <= med <= fm[a + 1] and fm[a + 1] > fm[a]:
            f = (np.log(med) - np.log(fm[a])) / (np.log(fm[a + 1]) - np.log(fm[a]))
            fc = float(np.exp(np.log(fcs[a]) + f * (np.log(fcs[a + 1]) - np.log(fcs[a]))))
    info = {"lambda": float(hi), "median": med, "p99": float(np.percentile(E[rows, j], 99)), "cost": cost,
            "fixed_cost_at_equal_median": fc, "bound_gain": (fc / cost) if fc else None}
    return th[j].astype(np.float32), info


def training_set(pos, vel, eps, thetas=DEFAULT_GRID, target=5e-4, samples_per_group=8, max_groups=8192, seed=0,
                 nleaf=16, ncrit=64, level_split=5, device=0, labels="crossing"):
    """(features, label theta, error table) for a random subset of groups.
    labels = "crossing": the angle at which the group's error reaches the
    target; "allocation": the cost-optimal allocation (allocation_labels)."""
    F, E, C, sizes = training_tables(pos, vel, eps, thetas, samples_per_group, max_groups, seed, nleaf, ncrit,
                                     level_split, device)
    if labels == "allocation":
        y, _ = allocation_labels(E, C, sizes, thetas, target)
    else:
        y = crossing_labels(E, thetas, target)
    return F, y, E


def calibrate(pos, vel, w, eps, target, fraction=0.9, samples=2048, iters=10, nleaf=16, ncrit=64, level_split=5,
              seed=0, device=0):
    """Scale c of the network's angle range (every group's angle becomes c
    times the network's), found by bisection on log c so that the median
    |da|/|a| of the system (pos, vel) against the FP64 direct sum is
    fraction * target.  Returns (c, lo * c, hi * c, median error at c).  The
    network's raw output sits below the target by design (its loss penalises
    too-large angles more); this one scalar moves it onto the target on a
    training system."""
    n = pos.shape[0]
    t = Treecode(eps=eps, theta=0.5, ncrit=ncrit, nleaf=nleaf, level_split=level_split, device=device)
    try:
        t.alloc(n)
        t.h_ptclPos[:] = pos
        t.h_ptclVel[:] = vel
        t.ptcl_h2d()
        rng = np.random.default_rng(seed)
        samp = np.ascontiguousarray(np.sort(rng.choice(n, min(samples, n), replace=False)).astype(np.int32))
        ref = t.direct_fp64(samp, include_self=True)
        refn = np.linalg.norm(ref[:, :3], axis=1)
        set_weights(t, w)
        t.buildTree(nleaf)
        t.computeMultipoles()
        t.makeGroups(level_split, ncrit)

        def median_err(c):
            set_theta_mode(t, 1, LO * c, HI * c)
            t.computeForces(False)
            acc = t.get_acc()[samp].astype(np.float64)
            return float(np.median(np.linalg.norm(acc[:, :3] - ref[:, :3], axis=1) / refn))

        goal = fraction * target
        lo_c, hi_c = 0.5, 2.0
        e_lo, e_hi = median_err(lo_c), median_err(hi_c)
        if e_lo > goal:
            return lo_c, LO * lo_c, HI * lo_c, e_lo
        if e_hi < goal:
            return hi_c, LO * hi_c, HI * hi_c, e_hi
        for _ in range(iters):
            mid = float(np.sqrt(lo_c * hi_c))
            if median_err(mid) > goal:
                hi_c = mid
            else:
                lo_c = mid
        return lo_c, LO * lo_c, HI * lo_c, median_err(lo_c)
    finally:
        t.close()
