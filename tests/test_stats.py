"""The Gamma-method error of jaxqft_b200.stats against the reference's own
estimator (tests/golden/golden_stats.json, written by make_golden_stats.py from
jaxqft/stats/autocorr.py) on seeded AR(1) series, and the agreement test of
jaxqft/testing/mcmc_smoke.py:135-145."""

import json
import os
import sys

import numpy as np

from jaxqft_b200.stats import compare_means, gamma_error
from tests.conftest import GOLDEN

sys.path.insert(0, GOLDEN)
from make_golden_stats import series  # noqa: E402


def test_gamma_error_matches_reference():
    with open(os.path.join(GOLDEN, "golden_stats.json")) as f:
        rows = json.load(f)
    for r in rows:
        e = gamma_error(series(r["n"], r["phi"], r["seed"]))
        assert e["window"] == r["window"], r
        assert abs(e["tau_int"] - r["tau_int"]) < 1e-12 * max(1.0, r["tau_int"]), (e, r)
        assert abs(e["sigma_mean"] - r["sigma_mean"]) < 1e-12 * r["sigma_mean"], (e, r)


def test_compare_means():
    a = series(2000, 0.5, 11)
    b = series(2000, 0.5, 12)
    assert compare_means(a, b)["agree"]
    assert not compare_means(a, b + 0.01)["agree"]
    c = compare_means(np.full(10, 0.5), np.full(10, 0.5))
    assert c["agree"] and c["sigma"] == 0.0
