"""Learned per-group opening bounds: training-set generation, training and
use of the 16 -> 64 -> 64 -> 1 network of csrc/learned.cu.

The learned form walks in the relative accuracy mode: a cell that passes the
geometric test at the safety angle theta_bound is still opened when its
octupole truncation error M l^3 / ds^5 exceeds the group's bound
tau_g = A_g 10^y_g, A_g being the group's mean |a| of the previous force
evaluation and y_g the network's output.  Training pairs come from the walk
and the FP64 direct sum, both on the GPU: for a random subset of groups and a
few particles in each, the walk runs with every group at each y of a grid
(theta mode 2 with host bounds), giving each group's error (geometric mean
over its sampled particles of |da|/|a| against the direct sum) and cost
(interaction counts) per y; the label is the cost-optimal y for the error
budget (allocation_labels), or the y at which the group's error reaches the
target.  The network is trained with the library's
own forward/backward kernels (bonsai_mlp_train, Adam, full batch) and used in
theta mode 1, where a feature kernel and an FP16-weight inference kernel set
each group's bound inside the step.  calibrate_relative then shifts the
output range by one constant so that the median error on a training system
is a chosen fraction of the target.

The per-group geometric angle (theta mode 2 without bounds) stays available;
training_tables / allocation_labels analyse it.
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import BonsaiError, load
from .treecode import Treecode, _check, _p

NFEAT = 16
NWEIGHTS = 5313
# output range of the per-group angle (geometric per-group analysis)
LO, HI, OVER = 0.25, 1.25, 3.0
# the learned form: output range of y = log10(tau / A), the safety angle, the
# grid of y the training tables cover, and the bound of the walk that
# precedes feature extraction in the tables
YLO, YHI = -4.0, -0.5
THETA_BOUND = 2.0
Y_GRID = tuple(np.round(np.arange(-3.6, -0.79, 0.2), 2))
ALPHA0 = 1e-2


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


def set_theta_mode(t: Treecode, mode: int, lo=None, hi=None):
    """0: fixed angle; 1: the learned form (lo, hi: output range of
    y = log10(tau / A), default (YLO, YHI)); 2: per-group angles and bounds
    from the host; 3: relative mode with one parameter alpha = lo."""
    if lo is None:
        lo, hi = (YLO, YHI) if mode == 1 else (LO, HI)
    if hi is None:
        hi = lo
    _check(t._L.bonsai_set_theta_mode(t.handle, mode, lo, hi), "set_theta_mode")


def set_relative_bound(t: Treecode, theta_bound: float):
    _check(t._L.bonsai_set_relative_bound(t.handle, float(theta_bound)), "set_relative_bound")


def set_group_tau(t: Treecode, tau):
    if tau is None:
        _check(t._L.bonsai_set_group_tau(t.handle, None, 0), "set_group_tau")
        return
    tau = np.ascontiguousarray(tau, np.float32)
    _check(t._L.bonsai_set_group_tau(t.handle, _p(tau), tau.shape[0]), "set_group_tau")


def group_scale(t: Treecode) -> np.ndarray:
    """A_g of the current groups (mean |a| of the previous evaluation)."""
    G = t.tree_info()["ngroups"]
    out = np.empty(max(G, 1), np.float32)
    _check(t._L.bonsai_get_group_scale(t.handle, _p(out)), "get_group_scale")
    return out[:G]


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


# ---------------------------------------------------------------------------
# the learned form: relative accuracy mode
# ---------------------------------------------------------------------------
def _prepare_relative(t: Treecode, nleaf, ncrit, level_split, alpha0, theta_bound, learned=None):
    """A relative walk at alpha0 (theta mode 2 with host bounds alpha0 A_g,
    after the fixed-angle first evaluation that gives A_g) so that acc and the
    walk statistics are those of a relative walk, then the tree rebuilt from
    the same positions (same groups, identity permutation): the state the
    learned features see inside a run.  learned = (weights, lo, hi): instead,
    the learned walk itself at its steady state (the fallback, then six
    evaluations), so that the features are those the network sees in a run."""
    set_relative_bound(t, theta_bound)
    if learned is not None:
        w, lo, hi = learned
        set_weights(t, w)
        set_theta_mode(t, 1, lo, hi)
        run_relative(t, nleaf, ncrit, level_split, evaluations=7)
        t.buildTree(nleaf)
        t.computeMultipoles()
        t.makeGroups(level_split, ncrit)
        return
    set_theta_mode(t, 0)
    t.buildTree(nleaf)
    t.computeMultipoles()
    t.makeGroups(level_split, ncrit)
    t.computeForces(False)
    t.buildTree(nleaf)
    t.computeMultipoles()
    t.makeGroups(level_split, ncrit)
    group_features(t)  # computes A_g from the previous accelerations
    A = group_scale(t).astype(np.float64)
    set_theta_mode(t, 2)
    set_group_theta(t, np.full(A.shape[0], theta_bound, np.float32))
    set_group_tau(t, (alpha0 * A).astype(np.float32))
    t.computeForces(False)
    set_group_tau(t, None)
    t.buildTree(nleaf)
    t.computeMultipoles()
    t.makeGroups(level_split, ncrit)


def relative_tables(pos, vel, eps, ys=Y_GRID, samples_per_group=8, max_groups=8192, seed=0, nleaf=16, ncrit=64,
                    level_split=5, alpha0=ALPHA0, theta_bound=THETA_BOUND, device=0, learned=None):
    """For a random subset of groups: features F (g, 16) as the learned walk
    sees them; the group scale A (g,); error table E (g, k) = geometric mean
    over the group's sampled particles of |da|/|a| against the FP64 direct sum
    with every group at tau = A 10^ys[k]; cost table C (g, k) = 64 n_approx +
    20 n_direct; group sizes (g,)."""
    n = pos.shape[0]
    t = Treecode(eps=eps, theta=0.5, ncrit=ncrit, nleaf=nleaf, level_split=level_split, device=device)
    try:
        t.alloc(n)
        t.h_ptclPos[:] = pos
        t.h_ptclVel[:] = vel
        t.ptcl_h2d()
        _prepare_relative(t, nleaf, ncrit, level_split, alpha0, theta_bound, learned)
        F = group_features(t)
        A = group_scale(t).astype(np.float64)
        groups = t.groups()
        G = groups.shape[0]
        ids = t.walk_arrays()["ids"]
        rng = np.random.default_rng(seed)
        gsel = np.sort(rng.choice(G, min(max_groups, G), replace=False))
        spos, owner = [], []
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
        set_group_theta(t, np.full(G, theta_bound, np.float32))
        E = np.zeros((gsel.shape[0], len(ys)))
        C = np.zeros((gsel.shape[0], len(ys)))
        for j, y in enumerate(ys):
            set_group_tau(t, (A * 10.0 ** y).astype(np.float32))
            t.computeForces(False)
            acc = t.walk_arrays()["acc"][spos].astype(np.float64)
            err = np.linalg.norm(acc[:, :3] - ref[:, :3], axis=1) / refn
            le = np.log(np.maximum(err, 1e-30))
            E[:, j] = np.exp(np.bincount(owner, weights=le, minlength=gsel.shape[0]) /
                             np.bincount(owner, minlength=gsel.shape[0]))
            cnt = group_interactions(t)[gsel].astype(np.float64)
            C[:, j] = 64.0 * cnt[:, 0] + 20.0 * cnt[:, 1]
        set_group_tau(t, None)
        return F[gsel], A[gsel], E, C, groups[gsel, 1].astype(np.float64)
    finally:
        t.close()


def relative_training_set(pos, vel, eps, target, ys=Y_GRID, labels="allocation", **kw):
    """(features, label y, error table) pairs.  labels = "allocation": the
    cost-optimal per-group y for a geometric-mean error of 0.9 * target
    (allocation_labels on the y grid: where a group's cost falls faster than
    its error grows it gets a larger y); "crossing": the y at which the
    group's own error reaches the target (every group equally accurate)."""
    F, A, E, C, sizes = relative_tables(pos, vel, eps, ys=ys, **kw)
    if labels == "allocation":
        y, _ = allocation_labels(E, C, sizes, ys, target)
    else:
        y = crossing_labels(E, ys, target)
    return F, y, E


def run_relative(t: Treecode, nleaf, ncrit, level_split, evaluations=3):
    """Force evaluations at the current positions: the first one after
    loading is the fixed-angle fallback; the later ones use the previous
    evaluation's accelerations and statistics, as inside a run."""
    for _ in range(evaluations):
        t.buildTree(nleaf)
        t.computeMultipoles()
        t.makeGroups(level_split, ncrit)
        t.computeForces(False)


def calibrate_relative(pos, vel, w, eps, target, fraction=0.9, samples=2048, iters=10, nleaf=16, ncrit=64,
                       level_split=5, theta_bound=THETA_BOUND, seed=0, device=0):
    """Shift c of the network's output range ((YLO + c, YHI + c)), found by
    bisection so that the median |da|/|a| of the system (pos, vel) against the
    FP64 direct sum is fraction * target.  Returns (c, lo, hi, median error)."""
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
        set_relative_bound(t, theta_bound)

        def median_err(c):
            set_theta_mode(t, 1, YLO + c, YHI + c)
            run_relative(t, nleaf, ncrit, level_split, evaluations=4)
            acc = t.get_acc()[samp].astype(np.float64)
            return float(np.median(np.linalg.norm(acc[:, :3] - ref[:, :3], axis=1) / refn))

        goal = fraction * target
        lo_c, hi_c = -1.5, 1.5
        e_lo, e_hi = median_err(lo_c), median_err(hi_c)
        if e_lo > goal:
            return lo_c, YLO + lo_c, YHI + lo_c, e_lo
        if e_hi < goal:
            return hi_c, YLO + hi_c, YHI + hi_c, e_hi
        for _ in range(iters):
            mid = 0.5 * (lo_c + hi_c)
            if median_err(mid) > goal:
                hi_c = mid
            else:
                lo_c = mid
        return lo_c, YLO + lo_c, YHI + lo_c, median_err(lo_c)
    finally:
        t.close()
