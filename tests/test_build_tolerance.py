"""The tolerance of the build-quality comparison (CPU only)."""
import numpy as np

from tests.helpers import build_recall_tolerance


def test_one_graph_per_side_is_the_sampling_error_of_a_difference():
    tol = build_recall_tolerance([0.9], [0.9], 20000)
    assert np.isclose(tol, 2 * np.sqrt(2 * 0.9 * 0.1 / 20000))


def test_seed_spread_widens_the_tolerance():
    narrow = build_recall_tolerance([0.99, 0.99, 0.99], [0.99, 0.99, 0.99], 20000)
    wide = build_recall_tolerance([0.985, 0.995, 0.99], [0.99, 0.994, 0.986], 20000)
    assert wide > narrow
    r, d = np.array([0.985, 0.995, 0.99]), np.array([0.99, 0.994, 0.986])
    samp = 0.99 * 0.01 / 20000
    want = 2 * np.sqrt(samp / 3 + samp / 3 + r.var(ddof=1) / 3 + d.var(ddof=1) / 3)
    assert np.isclose(wide, want)
