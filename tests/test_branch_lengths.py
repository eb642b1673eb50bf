"""Parsimony starting times for the edit model (casphy_b200.branch_lengths)."""
import numpy as np
import pytest

from casphy_b200.branch_lengths import T_MAX, T_MIN, parsimony_start


def test_times_from_change_counts():
    # tips 0, 1, 2; node 3 = root (parent of 4 and tip 2); node 4 = parent of tips 0, 1
    edge = np.array([[3, 4], [4, 0], [4, 1], [3, 2]])
    states = np.array([[0, 0, 0, 0],     # node 3: four unedited sites
                       [0, 0, 5, -1]])   # node 4: two unedited sites
    changes = np.array([1, 1, 0, 2])
    t = parsimony_start(edge, states, changes, ntip=3, rate=2.0)
    want = -np.log1p(-np.array([1 / 4, 1 / 2, 0.5 / 2, 2 / 4])) / 2.0
    assert np.allclose(t, want)


def test_bounds_and_caps():
    edge = np.array([[2, 0], [2, 1]])
    states = np.array([[7, 7, 7]])      # no unedited site at the parent
    t = parsimony_start(edge, states, np.array([0, 50]), ntip=2)
    assert np.all(t >= T_MIN) and np.all(t <= T_MAX)
    assert np.isclose(t[1], -np.log1p(-0.95))


def test_rejects_bad_input():
    edge = np.array([[1, 0]])
    with pytest.raises(ValueError):
        parsimony_start(edge, np.zeros((1, 2)), np.array([1, 2]), ntip=1)
    with pytest.raises(ValueError):
        parsimony_start(edge, np.zeros((1, 2)), np.array([1]), ntip=2)
    with pytest.raises(ValueError):
        parsimony_start(edge, np.zeros((1, 2)), np.array([1]), ntip=1, rate=0.0)
