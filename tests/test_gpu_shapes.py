"""Every hop kernel shape the autotuner can choose, pinned with WL_FORCE_TUNE:
classic thread-per-site kernels with 1/2/4 RHS per thread, the RHS-in-lanes
kernel with 4/8/16 lanes per site and the tensor-core FP16 hop (last shape; FP32
engines run the 16-lane kernel for it).  Each shape must give the same operator
(FP32: 2e-6, FP16: 4e-3 of FP64) and batched solves that reach an FP64 true
residual <= 1e-10 and agree with standalone FP64 solves."""

import os

import numpy as np
import pytest

from oracle import wilson as W
from tests.conftest import rel

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("CUDA device required", allow_module_level=True)

from jaxqft_b200.lib import Engine, WilsonContext  # noqa: E402

SHAPES = ["1,128,1,0", "2,64,2,0", "4,64,4,0", "1,128,1,4", "1,128,1,8", "1,128,1,16", "1,128,1,16,0,1"]
TOLS = {"single": 2e-6, "half": 4e-3}


@pytest.fixture(scope="module")
def setup():
    shape = (4, 6, 4, 8)
    rng = np.random.default_rng(31)
    U = W.hot_links(rng, shape, 1, 0.2)
    bc = (1, 1, 1j, -1)
    ctx = WilsonContext(shape, bc=bc)
    gauge = ctx.gauge(torch.from_numpy(U[0]))
    return shape, U, bc, ctx, gauge, rng


@pytest.fixture
def forced(request):
    os.environ["WL_FORCE_TUNE"] = request.param
    yield request.param
    del os.environ["WL_FORCE_TUNE"]


@pytest.mark.parametrize("forced", SHAPES, indirect=True)
@pytest.mark.parametrize("inner", ["single", "half"])
def test_operator_per_shape(setup, forced, inner):
    shape, U, bc, ctx, gauge, rng = setup
    m = -0.25
    eng = Engine(ctx, gauge, 16, op="eo_normal", inner=inner)
    xe = W.project(W.gaussian_spinor(rng, shape, 1), 0)
    s = W.schur_even(U, xe, m, bc, normalized=True)
    ref = W.schur_even(U, s, m, bc, normalized=True, dag=True)
    out = eng.debug_apply(2, m, torch.from_numpy(xe[0])).cpu().numpy()
    assert rel(out, ref[0]) < TOLS[inner], (forced, inner)
    eng.close()
    eng = Engine(ctx, gauge, 16, op="normal", inner=inner)
    x = W.gaussian_spinor(rng, shape, 1)
    out = eng.debug_apply(4, m, torch.from_numpy(x[0])).cpu().numpy()
    assert rel(out, W.apply_normal(U, x, m, bc)[0]) < TOLS[inner], (forced, inner)
    eng.close()


@pytest.mark.parametrize("forced", SHAPES, indirect=True)
def test_batched_solve_per_shape(setup, forced):
    shape, U, bc, ctx, gauge, rng = setup
    n = 13  # not a multiple of any lane / RHS-block count
    masses = np.linspace(-0.3, 0.1, n)
    b = W.project(W.gaussian_spinor(rng, shape, n), 0)
    b[5] *= 1e-4
    eng = Engine(ctx, gauge, n, op="eo_normal", inner="half", tol=1e-10, maxiter=3000)
    eng.admit(np.arange(n), torch.from_numpy(b), masses)
    na = n
    while na:
        eng.step(8)
        _, na = eng.poll()
    for r in range(n):
        x, st = eng.retire(r)
        assert st["status"] == 2, (forced, r, st)
        x = x.cpu().numpy()
        s = W.schur_even(U, x[None], masses[r], bc, normalized=True)
        ax = W.schur_even(U, s, masses[r], bc, normalized=True, dag=True)[0]
        assert np.linalg.norm(b[r] - ax) / np.linalg.norm(b[r]) <= 1e-10, (forced, r)
    eng.close()


# (forced shape, slots): FP64 engines with fewer than four slots run the
# thread-per-site stencils; a fifth field 1 selects two threads per site
FP64_CASES = [("1,64,1,0,1", 1), ("1,128,1,0,1", 3), ("1,256,1,0,1", 1), ("1,128,1,0", 1), ("1,128,1,0", 3)]


@pytest.mark.parametrize("forced,nslots", FP64_CASES, indirect=["forced"])
def test_fp64_stencil_shapes(setup, forced, nslots):
    """Every FP64 iterated-stencil shape gives the FP64 operator to 1e-13 and
    solves to the FP64 true-residual tolerance."""
    shape, U, bc, ctx, gauge, rng = setup
    m = -0.25
    eng = Engine(ctx, gauge, nslots, op="eo_normal", inner="double")
    xe = W.project(W.gaussian_spinor(rng, shape, 1), 0)
    s = W.schur_even(U, xe, m, bc, normalized=True)
    ref = W.schur_even(U, s, m, bc, normalized=True, dag=True)
    out = eng.debug_apply(2, m, torch.from_numpy(xe[0])).cpu().numpy()
    assert rel(out, ref[0]) < 1e-13, forced
    eng.close()
    eng = Engine(ctx, gauge, nslots, op="normal", inner="double")
    x = W.gaussian_spinor(rng, shape, 1)
    out = eng.debug_apply(4, m, torch.from_numpy(x[0])).cpu().numpy()
    assert rel(out, W.apply_normal(U, x, m, bc)[0]) < 1e-13, forced
    eng.close()
    masses = np.linspace(-0.3, 0.1, nslots)
    b = W.project(W.gaussian_spinor(rng, shape, nslots), 0)
    eng = Engine(ctx, gauge, nslots, op="eo_normal", inner="double", tol=1e-10, maxiter=3000)
    eng.admit(np.arange(nslots), torch.from_numpy(b), masses)
    na = nslots
    while na:
        eng.step(8)
        _, na = eng.poll()
    for r in range(nslots):
        xr, st = eng.retire(r)
        assert st["status"] == 2, (forced, r, st)
        xr = xr.cpu().numpy()
        s = W.schur_even(U, xr[None], masses[r], bc, normalized=True)
        ax = W.schur_even(U, s, masses[r], bc, normalized=True, dag=True)[0]
        assert np.linalg.norm(b[r] - ax) / np.linalg.norm(b[r]) <= 1e-10, (forced, r)
    eng.close()


# FP32 engines with fewer than four slots: thread-per-site and two-threads-per-site stencils
FP32_CASES = [("1,64,1,0,1", 1), ("1,128,1,0,1", 3), ("1,256,1,0,1", 1), ("1,128,1,0", 1), ("2,64,2,0", 3)]


@pytest.mark.parametrize("forced,nslots", FP32_CASES, indirect=["forced"])
def test_fp32_stencil_shapes(setup, forced, nslots):
    """Every FP32 iterated-stencil shape of a small engine (thread per site with 1 or 2 RHS,
    two threads per site) gives the operator within the FP32
    tolerance of the FP64 oracle, and its solves (FP64 reliable updates) reach an FP64 true
    residual <= 1e-10 and are bitwise reproducible."""
    shape, U, bc, ctx, gauge, rng = setup
    m = -0.25
    eng = Engine(ctx, gauge, nslots, op="eo_normal", inner="single")
    xe = W.project(W.gaussian_spinor(rng, shape, 1), 0)
    s = W.schur_even(U, xe, m, bc, normalized=True)
    ref = W.schur_even(U, s, m, bc, normalized=True, dag=True)
    out = eng.debug_apply(2, m, torch.from_numpy(xe[0])).cpu().numpy()
    assert rel(out, ref[0]) < TOLS["single"], forced
    eng.close()
    eng = Engine(ctx, gauge, nslots, op="normal", inner="single")
    x = W.gaussian_spinor(rng, shape, 1)
    for stage, ref in ((4, W.apply_normal(U, x, m, bc)[0]), (3, W.apply_D(U, x, m, bc)[0])):
        out = eng.debug_apply(stage, m, torch.from_numpy(x[0])).cpu().numpy()
        assert rel(out, ref) < TOLS["single"], (forced, stage)
    eng.close()
    masses = np.linspace(-0.3, 0.1, nslots)
    b = W.gaussian_spinor(rng, shape, nslots)
    for op in ("eo_normal", "normal"):
        bb = W.project(b, 0) if op == "eo_normal" else b
        runs = []
        for _ in range(2):
            eng = Engine(ctx, gauge, nslots, op=op, inner="single", tol=1e-10, maxiter=3000)
            eng.admit(np.arange(nslots), torch.from_numpy(bb), masses)
            na = nslots
            while na:
                eng.step(8)
                _, na = eng.poll()
            xs = []
            for r in range(nslots):
                xr, st = eng.retire(r)
                assert st["status"] == 2, (forced, op, r, st)
                xs.append(xr.cpu().numpy())
            eng.close()
            runs.append(xs)
        for r in range(nslots):
            assert np.array_equal(runs[0][r], runs[1][r]), (forced, op, r)
            xr = runs[0][r]
            if op == "eo_normal":
                s = W.schur_even(U, xr[None], masses[r], bc, normalized=True)
                ax = W.schur_even(U, s, masses[r], bc, normalized=True, dag=True)[0]
            else:
                ax = W.apply_normal(U, xr[None], masses[r], bc)[0]
            assert np.linalg.norm(bb[r] - ax) / np.linalg.norm(bb[r]) <= 1e-10, (forced, op, r)


@pytest.fixture
def forced_update(request):
    os.environ["WL_FORCE_UPDATE_TUNE"] = request.param
    yield request.param
    del os.environ["WL_FORCE_UPDATE_TUNE"]


@pytest.mark.parametrize("forced_update", ["16", "8", "4", "8,2", "4,2", "4,4"], indirect=True)
def test_update_hop_shapes(setup, forced_update):
    """Every shape of the FP64 reliable-update hop (RHS lanes per group, groups a block
    works through on its staged links) gives solves that reach the FP64 true-residual
    tolerance, checked against the oracle operator."""
    shape, U, bc, ctx, gauge, rng = setup
    n = 13
    masses = np.linspace(-0.3, 0.1, n)
    b = W.project(W.gaussian_spinor(rng, shape, n), 0)
    eng = Engine(ctx, gauge, n, op="eo_normal", inner="half", tol=1e-10, maxiter=3000)
    eng.admit(np.arange(n), torch.from_numpy(b), masses)
    na = n
    while na:
        eng.step(8)
        _, na = eng.poll()
    for r in range(n):
        x, st = eng.retire(r)
        assert st["status"] == 2, (forced_update, r, st)
        x = x.cpu().numpy()
        s = W.schur_even(U, x[None], masses[r], bc, normalized=True)
        ax = W.schur_even(U, s, masses[r], bc, normalized=True, dag=True)[0]
        assert np.linalg.norm(b[r] - ax) / np.linalg.norm(b[r]) <= 1e-10, (forced_update, r)
    eng.close()
