"""Golden outputs of the reference's Gamma-method error (jaxqft/stats/autocorr.py).

Loads that file by path (it needs only numpy) and records, for seeded AR(1)
series of several lengths and correlations, tau_int, the window and the error
of the mean, in ``golden_stats.json`` beside this script.  Usage:
    python tests/golden/make_golden_stats.py --ref /path/to/jaxQFT
"""

from __future__ import annotations

import argparse
import importlib.util
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = [(200, 0.0, 1), (200, 0.5, 2), (1000, 0.9, 3), (64, 0.7, 4), (500, -0.3, 5)]


def series(n, phi, seed):
    """AR(1): x_t = phi x_{t-1} + e_t, seeded numpy PCG64."""
    rng = np.random.default_rng(seed)
    e = rng.standard_normal(n)
    x = np.empty(n)
    x[0] = e[0]
    for t in range(1, n):
        x[t] = phi * x[t - 1] + e[t]
    return 0.55 + 0.01 * x


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="root of the jaxQFT source tree")
    args = ap.parse_args()
    spec = importlib.util.spec_from_file_location("autocorr", os.path.join(args.ref, "jaxqft", "stats", "autocorr.py"))
    ac = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(ac)
    rows = []
    for n, phi, seed in CASES:
        r = ac.integrated_autocorr_time(series(n, phi, seed), method="gamma")
        rows.append({"n": n, "phi": phi, "seed": seed, "tau_int": r["tau_int"], "window": r["window"],
                     "sigma_mean": r["sigma_mean"], "ess": r["ess"]})
    with open(os.path.join(HERE, "golden_stats.json"), "w") as f:
        json.dump(rows, f, indent=1)
    print(f"wrote {len(rows)} rows")


if __name__ == "__main__":
    main()
