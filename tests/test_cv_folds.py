"""Fold rules of the cross-validation and its score, on the CPU, against the reference's
own functions' outputs (tests/golden/cv_proj.npz)."""
import numpy as np

from adamixture_b200.src import cv
from oracle import solvers as osv


def test_shuffled_list_rule_matches_reference(cv_proj):
    G = cv_proj["G"]
    flat = np.flatnonzero(G != 3)
    np.testing.assert_array_equal(cv.shuffle_observed(flat, 42), cv_proj["cv_shuffled"])


def test_hash_rule_matches_reference(cv_proj):
    probe = cv_proj["hash_probe"]
    got = np.stack([cv.hash_fold_mask(probe, 42, 5, f) for f in range(5)])
    assert (got.sum(0) == 1).all()
    np.testing.assert_array_equal(got.argmax(0), cv_proj["hash_fold"])


def test_deviance_oracle_matches_a_direct_sum():
    rng = np.random.default_rng(1)
    G = rng.choice(4, size=(13, 11), p=[0.3, 0.3, 0.3, 0.1]).astype(np.uint8)
    P = rng.uniform(0.01, 0.99, (13, 2))
    Q = rng.dirichlet([1, 1], 11)
    flat = rng.choice(13 * 11, 40, replace=False)
    want = 0.0
    for f in flat:
        j, i = divmod(int(f), 11)
        g = float(G[j, i])
        if g == 3:
            continue
        mu = min(max(2.0 * float(P[j] @ Q[i]), 1e-10), 2 - 1e-10)
        want += (g * np.log(g / mu) if g > 0 else 0.0) + ((2 - g) * np.log((2 - g) / (2 - mu)) if g < 2 else 0.0)
    assert abs(osv.deviance_sum(G, P, Q, flat) - want) <= 1e-12 * abs(want)
