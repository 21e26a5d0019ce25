"""Host-side label logic of the learned opening angles (no GPU)."""
import numpy as np

from bonsai2_b200 import learned as Lr

TH = np.round(np.arange(0.3, 1.2501, 0.05), 2)


def _tables(slopes, costs, n_each=200):
    # error e_g(theta) = 1e-4 * (theta / 0.5) ** slope_g, cost c_g(theta) = c_g * (0.5 / theta) ** 2
    E, C = [], []
    for s, c in zip(slopes, costs):
        for _ in range(n_each):
            E.append(1e-4 * (TH / 0.5) ** s)
            C.append(c * (0.5 / TH) ** 2)
    return np.array(E), np.array(C), np.full(len(E), 32.0)


def test_crossing_labels_interpolate_in_log_error():
    E = np.array([1e-4 * (TH / 0.5) ** 4])
    y = Lr.crossing_labels(E, TH, 1e-3)
    want = 0.5 * 10 ** 0.25  # 1e-4 * (t/0.5)^4 = 1e-3
    assert abs(y[0] - want) < 0.01


def test_allocation_equal_groups_matches_fixed_angle():
    E, C, w = _tables([4, 4], [1.0, 1.0])
    y, info = Lr.allocation_labels(E, C, w, TH, 1e-3)
    assert np.all(y == y[0])
    assert info["median"] <= 0.9e-3 * 1.0001
    assert 0.95 < info["bound_gain"] < 1.05


def test_allocation_gains_on_unequal_groups():
    # groups that lose accuracy slowly with the angle should get larger angles
    E, C, w = _tables([2, 3, 4, 5, 6], [1.0] * 5)
    y, info = Lr.allocation_labels(E, C, w, TH, 1e-3)
    assert y[:200].mean() > y[800:].mean()
    assert info["bound_gain"] > 1.05
