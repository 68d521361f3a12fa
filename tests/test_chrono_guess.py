"""Chronological initial guesses of the drop-in theory (last / polynomial /
minimal-residual extrapolation) against the reference's own predictors
(golden_chrono.npz from jaxqft/models/su3_wilson_nf2.py:85-194).  The
predictors are plain tensor algebra, so this runs on CPU torch tensors; on the
GPU the same code runs on device tensors."""

import numpy as np
import torch

from jaxqft_b200.su3_wilson_nf2 import _chrono_predict, _chrono_predict_mre
from tests.conftest import load_golden, rel


def _t(a):
    return torch.from_numpy(np.ascontiguousarray(a))


def test_polynomial_and_last_match_reference():
    g = load_golden("chrono")
    xs = [_t(x) for x in g["xs"]]
    assert rel(_chrono_predict(xs, "poly", 4).numpy(), g["poly"]) < 1e-14
    assert rel(_chrono_predict(xs, "poly", 3).numpy(), g["poly3"]) < 1e-14
    assert rel(_chrono_predict(xs, "last", 4).numpy(), g["last"]) < 1e-15


def test_mre_matches_reference_and_falls_back():
    g = load_golden("chrono")
    xs, ys = [_t(x) for x in g["xs"]], [_t(y) for y in g["ys"]]
    x0 = _chrono_predict_mre(xs, ys, _t(g["target"]))
    assert rel(x0.numpy(), g["mre"]) < 1e-12
    assert np.linalg.norm(g["mre"] - g["last"]) > 0.1  # the golden case exercises acceptance
    far = _chrono_predict_mre(xs, ys, _t(g["far"]))
    assert rel(far.numpy(), g["mre_far"]) < 1e-15  # rejected -> last solution
