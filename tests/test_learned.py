"""Learned per-group opening criteria.

CPU: the numpy restatement of the network (oracle/mlp_oracle.py) has a
gradient that matches finite differences.  GPU: the CUDA forward/backward
kernels match the numpy gradient; a per-group walk whose angles all equal the
fixed angle reproduces the fixed walk bit for bit; the relative modes fall
back to the fixed walk, bit for bit, while there are no previous
accelerations, and the FP64 checker walk takes their interaction lists;
training lowers the loss; and, on a Plummer sphere the network was neither
trained nor calibrated on, the learned form costs fewer interactions than
the fixed angle that reaches the same median force error (the metric's
statistic).
"""
import numpy as np
import pytest

LO, HI, OVER = 0.25, 1.25, 3.0


def _data(S=300, seed=0):
    rng = np.random.default_rng(seed)
    X = rng.normal(size=(S, 16)).astype(np.float32)
    y = rng.uniform(0.3, 1.1, S).astype(np.float32)
    return X, y


def test_oracle_gradient_finite_differences():
    from oracle import mlp_oracle as M
    from bonsai2_b200.learned import init_weights
    X, y = _data(60)
    w = init_weights(1).astype(np.float64)
    _, g = M.loss_grad(X, y, w, LO, HI, OVER)
    for idx in [0, 511, 1087, 3000, 5200, 5250, 5312]:
        e = 1e-6
        wp, wm = w.copy(), w.copy()
        wp[idx] += e
        wm[idx] -= e
        fd = (M.loss_grad(X, y, wp, LO, HI, OVER)[0] - M.loss_grad(X, y, wm, LO, HI, OVER)[0]) / (2 * e)
        assert abs(fd - g[idx]) <= 1e-6 * max(1.0, abs(fd))


@pytest.mark.gpu
def test_gpu_gradient_matches_oracle(lib):
    from oracle import mlp_oracle as M
    from bonsai2_b200 import learned as Lr
    X, y = _data(300)
    w = Lr.init_weights(2)
    loss, g = Lr.loss_grad(X, y, w)
    lo, go = M.loss_grad(X, y, w.astype(np.float64), LO, HI, OVER)
    assert abs(loss - lo) <= 1e-5 * abs(lo)
    assert np.allclose(g, go, rtol=1e-3, atol=1e-6 * np.abs(go).max())
    # prediction = the oracle forward
    th = Lr.predict(X, w)
    to, _ = M.forward(X.astype(np.float64), w.astype(np.float64), LO, HI)
    assert np.allclose(th, to, atol=2e-5)


@pytest.mark.gpu
def test_training_lowers_loss(lib):
    from bonsai2_b200 import learned as Lr
    rng = np.random.default_rng(3)
    X = rng.normal(size=(2000, 16)).astype(np.float32)
    y = (0.6 + 0.2 * np.tanh(X[:, 0] - 0.5 * X[:, 3])).astype(np.float32)
    w0 = Lr.init_weights(0)
    l0, _ = Lr.loss_grad(X, y, w0)
    w, l1 = Lr.train(X, y, w0, epochs=400, lr=3e-3)
    assert l1 < 0.2 * l0
    w2, l2 = Lr.train(X, y, w0, epochs=400, lr=3e-3)
    assert np.array_equal(w, w2) and l1 == l2  # deterministic


@pytest.mark.gpu
def test_pergroup_theta_equal_to_fixed_is_exact(oracle, lib):
    import bonsai2_b200 as B
    from bonsai2_b200 import learned as Lr
    pos, vel = oracle.plummer_float4(30000, 4)
    out = []
    for mode in (0, 2):
        t = B.Treecode(eps=0.01, theta=0.55)
        t.alloc(pos.shape[0])
        t.h_ptclPos[:] = pos
        t.h_ptclVel[:] = vel
        t.ptcl_h2d()
        t.buildTree(16)
        t.computeMultipoles()
        t.makeGroups(5, 64)
        if mode == 2:
            Lr.set_theta_mode(t, 2)
            Lr.set_group_theta(t, np.full(t.tree_info()["ngroups"], 0.55, np.float32))
        stats = t.computeForces(True)
        out.append((t.get_acc(), stats))
        t.close()
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])


def _interp_cost(points, e):
    """Cost of the fixed angle whose error equals e, interpolated in log-log
    between the sweep points (angle, error, cost) bracketing e."""
    pts = sorted(points, key=lambda p: p[1])
    for (t0, e0, c0), (t1, e1, c1) in zip(pts, pts[1:]):
        if e0 <= e <= e1 and e1 > e0:
            f = (np.log(e) - np.log(e0)) / (np.log(e1) - np.log(e0))
            return float(np.exp(np.log(c0) + f * (np.log(c1) - np.log(c0))))
    return None


def _load(B, pos, vel, theta=0.6, eps=0.01):
    t = B.Treecode(eps=eps, theta=theta)
    t.alloc(pos.shape[0])
    t.h_ptclPos[:] = pos
    t.h_ptclVel[:] = vel
    t.ptcl_h2d()
    return t


def _evaluate(t):
    t.buildTree(16)
    t.computeMultipoles()
    t.makeGroups(5, 64)
    return t.computeForces(True)


@pytest.mark.gpu
def test_relative_modes_fall_back_to_fixed_angle(oracle, lib):
    """Without previous accelerations (the first evaluation after loading)
    the learned and single-parameter relative modes walk at the fixed angle:
    accelerations and statistics bit-identical to theta mode 0.  The next
    evaluation uses the relative test and opens more cells than the
    geometric test at the safety angle alone."""
    import bonsai2_b200 as B
    from bonsai2_b200 import learned as Lr
    pos, vel = oracle.plummer_float4(30000, 5)
    t = _load(B, pos, vel)
    s0 = _evaluate(t)
    a0 = t.get_acc()
    t.close()
    for mode in (1, 3):
        t = _load(B, pos, vel)
        if mode == 1:
            Lr.set_weights(t, Lr.init_weights(3))
            Lr.set_theta_mode(t, 1, Lr.YLO, Lr.YHI)
        else:
            Lr.set_theta_mode(t, 3, 1e-2, 1e-2)
        s1 = _evaluate(t)
        assert np.array_equal(t.get_acc(), a0) and np.array_equal(s1, s0), mode
        s2 = _evaluate(t)   # now with the previous accelerations
        assert Lr.group_scale(t).min() > 0
        t.close()
        # the geometric test alone at the safety angle
        g = _load(B, pos, vel, theta=Lr.THETA_BOUND)
        sg = _evaluate(g)
        g.close()
        assert s2[2] > sg[2], (mode, s2, sg)


@pytest.mark.gpu
def test_learned_form_starts_with_the_single_alpha_bound(oracle, lib):
    """The evaluation after the fixed-angle fallback reads statistics of a
    walk without the relative test, which the network never saw in training:
    it takes the single-parameter bound tau = 1e-2 A_g instead (the state the
    training tables are recorded after), so its accelerations equal theta
    mode 3's at alpha 1e-2 bit for bit, whatever the weights; the evaluation
    after it uses the network."""
    import bonsai2_b200 as B
    from bonsai2_b200 import learned as Lr
    pos, vel = oracle.plummer_float4(30000, 7)
    accs = {}
    for mode in (1, 3):
        t = _load(B, pos, vel)
        Lr.set_relative_bound(t, Lr.THETA_BOUND)
        if mode == 1:
            Lr.set_weights(t, Lr.init_weights(5))
            Lr.set_theta_mode(t, 1, Lr.YLO, Lr.YHI)
        else:
            Lr.set_theta_mode(t, 3, Lr.ALPHA0, Lr.ALPHA0)
        _evaluate(t)   # fixed-angle fallback
        s2 = _evaluate(t)
        a2 = t.get_acc()
        s3 = _evaluate(t)
        accs[mode] = (a2, s2, s3)
        t.close()
    assert np.array_equal(accs[1][0], accs[3][0]) and np.array_equal(accs[1][1], accs[3][1])
    assert not np.array_equal(accs[1][2], accs[3][2])   # then the network's own bounds


@pytest.mark.gpu
def test_relative_mode_fp64_checker_takes_the_same_lists(oracle, lib):
    import bonsai2_b200 as B
    from bonsai2_b200 import learned as Lr
    pos, vel = oracle.plummer_float4(20000, 6)
    t = _load(B, pos, vel)
    Lr.set_theta_mode(t, 3, 3e-3, 3e-3)
    _evaluate(t)
    st = _evaluate(t)
    acc64, st64 = t.compute_forces_fp64()
    t.close()
    n = pos.shape[0]
    assert abs(st64[0] / n - st[2]) < 1e-9 and abs(st64[1] / n - st[0]) < 1e-9, (st, st64)


def _interp_cost(points, e):
    """Cost of the fixed angle whose error equals e, interpolated in log-log
    between the sweep points (angle, error, cost) bracketing e."""
    pts = sorted(points, key=lambda p: p[1])
    for (t0, e0, c0), (t1, e1, c1) in zip(pts, pts[1:]):
        if e0 <= e <= e1 and e1 > e0:
            f = (np.log(e) - np.log(e0)) / (np.log(e1) - np.log(e0))
            return float(np.exp(np.log(c0) + f * (np.log(c1) - np.log(c0))))
    return None


@pytest.mark.gpu
def test_learned_form_gains_at_equal_median(oracle, lib):
    """Trained and calibrated on one Plummer sphere, judged on another: the
    learned form meets the 1e-3 median bar and costs fewer model flops
    (20 per direct + 64 per approximate interaction) than the fixed angle of
    equal median error, interpolated over a sweep of fixed angles."""
    import bonsai2_b200 as B
    from bonsai2_b200 import learned as Lr
    n, eps, target = 1 << 19, 0.01, 1e-3
    ptr, vtr = B.plummer(n, 1001)      # training system
    X, y, _ = Lr.relative_training_set(ptr, vtr, eps=eps, target=target, max_groups=4096)
    w, loss = Lr.train(X, y, epochs=3000, lr=3e-3, lo=Lr.YLO, hi=Lr.YHI)
    c, lo, hi, e_cal = Lr.calibrate_relative(ptr, vtr, w, eps, target)
    pos, vel = B.plummer(n, 2002)      # evaluation system (neither trained nor calibrated on)
    rng = np.random.default_rng(9)
    samp = rng.choice(n, 2048, replace=False).astype(np.int32)
    ref = oracle.direct_fp64(pos, samp, eps)
    refn = np.linalg.norm(ref[:, :3], axis=1)

    def run(theta, learned):
        t = _load(B, pos, vel, theta=theta, eps=eps)
        if learned:
            Lr.set_weights(t, w)
            Lr.set_theta_mode(t, 1, lo, hi)
        for _ in range(7 if learned else 1):  # the learned bounds' steady state
            s = _evaluate(t)
        acc = t.get_acc().astype(np.float64)
        t.close()
        err = np.linalg.norm(acc[samp, :3] - ref[:, :3], axis=1) / refn
        return np.median(err), np.percentile(err, 99), 20 * s[0] + 64 * s[2]

    mL, pL, cL = run(0.6, True)
    sweep = [(th,) + run(th, False) for th in (0.5, 0.6, 0.7, 0.8, 0.9, 1.0, 1.1)]
    assert mL <= target
    c_eq = _interp_cost([(th, m, c) for th, m, p, c in sweep], mL)
    assert c_eq is not None, (mL, sweep)
    assert cL < c_eq / 1.1, (mL, pL, cL, c_eq, sweep)


@pytest.mark.gpu
def test_cost_optimal_allocation_beats_fixed_angle():
    """The cost-optimal per-group angles (allocation_labels on every group's
    error and cost tables) walk the same system at equal median error for
    less work than a fixed angle: measured in the walk's model flops from its
    interaction counts, so the result is deterministic."""
    import bonsai2_b200 as B
    from bonsai2_b200 import learned as Lr
    n = 1 << 18
    p, v = B.plummer(n, 21)
    F, E, C, sz = Lr.training_tables(p, v, eps=0.01, samples_per_group=8, max_groups=1 << 30)
    y, info = Lr.allocation_labels(E, C, sz, Lr.DEFAULT_GRID, 1e-3)
    assert info["bound_gain"] > 1.1
    # the same tables, read for the allocation and for every fixed angle: cost at equal median
    rows = np.arange(E.shape[0])
    j = np.abs(np.asarray(Lr.DEFAULT_GRID)[None, :] - y[:, None].astype(np.float64)).argmin(axis=1)
    med_alloc = Lr._wmedian(E[rows, j], sz)
    cost_alloc = C[rows, j].sum()
    fixed = [(Lr._wmedian(E[:, k], sz), C[:, k].sum()) for k in range(E.shape[1])]
    cheaper = [c for m, c in fixed if m <= med_alloc]
    assert cheaper and cost_alloc < 0.9 * min(cheaper)
    # and applied in a walk (theta mode 2), the counted work matches the tables
    t = B.Treecode(eps=0.01, theta=0.5)
    t.alloc(n)
    t.h_ptclPos[:] = p
    t.h_ptclVel[:] = v
    t.ptcl_h2d()
    t.buildTree(16)
    t.computeMultipoles()
    t.makeGroups(5, 64)
    Lr.set_theta_mode(t, 2)
    Lr.set_group_theta(t, y)
    t.computeForces(False)
    cnt = Lr.group_interactions(t).astype(np.float64)
    assert np.isclose((64.0 * cnt[:, 0] + 20.0 * cnt[:, 1]).sum(), cost_alloc, rtol=1e-9)
    t.close()
