"""The allocation-free Schur normal operator (wl_apply_schur_normal_noalloc).

Callers such as an XLA custom-call handler cannot call cudaMalloc (the
framework owns device memory); this entry point keeps its intermediates in a
static device array.  It must agree with the allocating entry point
wl_apply(WL_OP_SCHUR_E_NORMAL) -- same FP64 tolerance as the operator tests
(1e-13 relative) -- on two calls in a row (the scratch keeps the previous
call's contents), and must reject requests larger than its scratch.  Both
entry points run the same hop kernels, so the result is also checked against
the numpy oracle's S_e^dag S_e, normalized and unnormalized.  This file
is collected last so that a stop-at-first-failure run has run everything else.
"""

import ctypes

import numpy as np
import pytest

from oracle import wilson as W
from tests.conftest import rel

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("CUDA device required", allow_module_level=True)

from jaxqft_b200 import lib as L  # noqa: E402

TOL = 1e-13


def _noalloc(ctx, gauge, mass, x, normalized=True):
    out = torch.empty_like(x)
    rc = ctx.lib.wl_apply_schur_normal_noalloc(ctx.handle, gauge.handle, float(mass),
                                               L.FLAG_NORMALIZED if normalized else 0, x.data_ptr(),
                                               out.data_ptr(), x.numel() // (12 * ctx.volume))
    return rc, out


def test_noalloc_matches_allocating_entry_point_twice():
    shape = (8, 8, 8, 16)
    rng = np.random.default_rng(17)
    U = W.hot_links(rng, shape, 1, 0.2)
    m = -0.2962963
    bc = (1, 1, 1, -1)
    ctx = L.WilsonContext(shape, bc=bc)
    gauge = ctx.gauge(torch.from_numpy(U[0]))
    for call, nrhs in enumerate((2, 1)):  # two calls in a row, different inputs and sizes
        x = torch.from_numpy(W.project(W.gaussian_spinor(rng, shape, nrhs), 0)).cuda()
        ref = ctx.apply("SCHUR_E_NORMAL", gauge, m, x, normalized=True)
        rc, out = _noalloc(ctx, gauge, m, x)
        assert rc == L.WL_OK, ctx.lib.wl_last_error(ctx.handle)
        torch.cuda.synchronize()
        assert rel(out.cpu().numpy(), ref.cpu().numpy()) < TOL, call
        xn = x.cpu().numpy()
        orc = W.schur_even(U, W.schur_even(U, xn, m, bc, normalized=True), m, bc, normalized=True, dag=True)
        assert rel(out.cpu().numpy(), orc) < TOL, call
    # the unnormalized operator as well
    rc, out = _noalloc(ctx, gauge, m, x, normalized=False)
    ref = ctx.apply("SCHUR_E_NORMAL", gauge, m, x, normalized=False)
    assert rc == L.WL_OK and rel(out.cpu().numpy(), ref.cpu().numpy()) < TOL
    xn = x.cpu().numpy()
    orc = W.schur_even(U, W.schur_even(U, xn, m, bc), m, bc, dag=True)
    assert rel(out.cpu().numpy(), orc) < TOL


def test_noalloc_rejects_requests_beyond_its_scratch():
    shape = (8, 8, 8, 16)  # V = 8192: at most 21 fields fit in 64 MiB
    rng = np.random.default_rng(18)
    U = W.hot_links(rng, shape, 1, 0.2)
    ctx = L.WilsonContext(shape)
    gauge = ctx.gauge(torch.from_numpy(U[0]))
    x = torch.zeros((22, *shape, 4, 3), dtype=torch.complex128, device="cuda")
    rc, _ = _noalloc(ctx, gauge, 0.1, x)
    assert rc == L.WL_ERR_ARG
    assert b"scratch" in ctx.lib.wl_last_error(ctx.handle)
