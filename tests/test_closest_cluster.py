"""Cluster assignment of new queries for the Monte Carlo random-match model
(RandomMC::closest_cluster, src/random/random_match.cpp:222-227, 338-360),
a host-only C-ABI function (no GPU needed).  The reference's test databases
(test/small_mass*.h5) hold no /random group and its nearest_neighbour needs
Eigen, so no reference output pins this step: the oracle's C restatement and
an independent numpy one do."""
import numpy as np
import pytest

import oracle
from sketchlib_b200 import capi


def _restated(centroids, bases, use_rc):
    b = bases.copy()
    if use_rc:
        at = 0.5 * (b[:, 0] + b[:, 3])
        cg = 0.5 * (b[:, 1] + b[:, 2])
        b = np.stack([at, cg, cg, at], axis=1)
    d = ((centroids[None, :, :] - b.astype(np.float32)[:, None, :]) ** 2).sum(axis=2)
    return np.argmin(d, axis=1).astype(np.uint16)       # first minimum on ties


@pytest.mark.parametrize("use_rc", [True, False])
def test_matches_nearest_centroid(use_rc):
    rng = np.random.default_rng(17)
    centroids = rng.dirichlet(np.ones(4) * 10, 5).astype(np.float32)
    bases = rng.dirichlet(np.ones(4) * 10, 2000)
    got = capi.closest_cluster(centroids, bases, use_rc=use_rc)
    np.testing.assert_array_equal(got, _restated(centroids, bases, use_rc))
    np.testing.assert_array_equal(got, oracle.closest_cluster(centroids, bases, use_rc))
    assert len(np.unique(got)) > 1


def test_strand_folding_and_edges():
    centroids = np.array([[0.25, 0.25, 0.25, 0.25], [0.4, 0.1, 0.1, 0.4]], np.float32)
    # A-rich and T-rich genomes look the same once the strand is unknown
    a_rich = np.array([[0.7, 0.1, 0.1, 0.1]])
    t_rich = np.array([[0.1, 0.1, 0.1, 0.7]])
    assert capi.closest_cluster(centroids, a_rich)[0] == capi.closest_cluster(centroids, t_rich)[0] == 1
    assert capi.closest_cluster(centroids[:0], a_rich)[0] == 0          # no clusters: 0
    assert capi.closest_cluster(centroids, np.zeros((0, 4))).shape == (0,)
