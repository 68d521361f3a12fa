"""Monte Carlo error of a chain mean with autocorrelations (host side).

Mirrors the ``method="gamma"`` estimator of jaxqft/stats/autocorr.py:25-220,
which jaxqft/testing/mcmc_smoke.py:43-70 uses to put error bars on chain means
and :135-145 to decide whether two chains agree: the autocovariance Gamma(t) is
computed by FFT with the unbiased 1/(n - t) normalisation, the integrated
autocorrelation time tau(W) = 1/2 + sum_{t=1..W} Gamma(t)/Gamma(0) is summed
until the first W with W >= c tau(W) (U. Wolff, "Monte Carlo errors with less
errors", Comput. Phys. Commun. 156 (2004) 143, automatic windowing with the
reference's constant c = 5), and the variance of the mean is
(Gamma(0) + 2 sum_{t=1..W} Gamma(t)) / n.
"""

from __future__ import annotations

import math

import numpy as np


def gamma_error(x, c: float = 5.0) -> dict:
    """tau_int, effective sample size, window and sigma of the mean of series x."""
    a = np.asarray(x, dtype=np.float64).reshape(-1)
    n = a.size
    if n < 2:
        return {"mean": float(a.mean()) if n else float("nan"), "sigma_mean": float("nan"), "tau_int": float("nan"),
                "ess": float("nan"), "window": 0, "n": int(n)}
    y = a - a.mean()
    f = np.fft.rfft(y, n=2 * n)
    gam = np.fft.irfft(f * np.conj(f), n=2 * n)[:n] / np.arange(n, 0, -1, dtype=np.float64)
    g0 = float(gam[0])
    if not math.isfinite(g0) or g0 <= 0.0:  # a constant series: no spread, no error
        return {"mean": float(a.mean()), "sigma_mean": 0.0, "tau_int": 0.5, "ess": float(n), "window": 0,
                "n": int(n)}
    tau, w = 0.5, n - 1
    for t in range(1, n):
        tau = max(tau + float(gam[t]) / g0, 0.5)
        if t >= c * tau:
            w = t
            break
    var = (g0 + 2.0 * float(np.sum(gam[1:w + 1]))) / n
    sigma = math.sqrt(var) if var > 0.0 else float("nan")
    if not math.isfinite(sigma):  # fall back to the naive error scaled by the effective sample size
        sigma = float(np.std(a, ddof=1)) / math.sqrt(max(1.0, n / (2.0 * tau)))
    return {"mean": float(a.mean()), "sigma_mean": sigma, "tau_int": float(tau), "ess": float(n / (2.0 * tau)),
            "window": int(w), "n": int(n)}


def compare_means(a, b, sigma_cut: float = 4.0) -> dict:
    """|mean(a) - mean(b)| in units of the combined Gamma-method error
    (mcmc_smoke.py:135-145): the chains agree when sigma < sigma_cut."""
    ea, eb = gamma_error(a), gamma_error(b)
    d = abs(ea["mean"] - eb["mean"])
    comb = math.sqrt(ea["sigma_mean"] ** 2 + eb["sigma_mean"] ** 2)
    sigma = d / comb if comb > 0.0 else (0.0 if d == 0.0 else float("inf"))
    return {"a": ea["mean"], "b": eb["mean"], "err_a": ea["sigma_mean"], "err_b": eb["sigma_mean"], "delta": d,
            "sigma": sigma, "agree": bool(sigma < sigma_cut)}
