"""The flop counter of jaxqft_b200.wilson.WilsonDiracOperator against the
reference's own counts (tests/golden/golden_flops.json, written by
tests/golden/make_golden_flops.py from jaxqft/fermions/wilson.py:349-437) and
the golden 3600 flops/site of D stored with the operator fixtures."""

import json
import os

import pytest

from jaxqft_b200.wilson import WilsonDiracOperator
from tests.conftest import GOLDEN, load_golden


def test_flop_counts_match_reference_grid():
    with open(os.path.join(GOLDEN, "golden_flops.json")) as f:
        rows = json.load(f)
    op = WilsonDiracOperator(ndim=4)
    for r in rows:
        assert op.flops_per_site_dslash(r["nc"], use_sparse_gamma=r["sparse"]) == r["dslash"], r
        assert op.flops_per_site_matvec(r["nc"], use_sparse_gamma=r["sparse"], include_diagonal=r["diag"]) == r["matvec"]
        assert op.flops_per_matvec_call(r["nc"], 4096, 2, use_sparse_gamma=r["sparse"],
                                        include_diagonal=r["diag"]) == r["call_V4096_B2"]


def test_flops_per_site_D_is_3600():
    assert WilsonDiracOperator().flops_per_site_matvec(nc=3) == int(load_golden("a")["ref_flops_site_D"])
    assert WilsonDiracOperator().flops_per_site_dslash(nc=3) == 3552


def test_flop_counter_rejects_bad_nc():
    with pytest.raises(ValueError):
        WilsonDiracOperator().flops_per_site_dslash(nc=0)
    with pytest.raises(ValueError):
        WilsonDiracOperator(ndim=0)
