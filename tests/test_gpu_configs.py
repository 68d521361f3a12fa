"""Full-size cases of the measured configurations, on the GPU.

C2: 16^3x32, links exp(i*0.2*H), kappa 0.135, antiperiodic t, one Gaussian RHS.
    The EO normal system solved with FP32 and with FP16 iterated operators (FP64
    reliable updates) reaches an FP64 true residual <= 1e-10 and agrees with
    plain FP64 CG on the same system.
C3: 24^3x48, kappa 0.130 (the second kappa of the batched configuration), 16
    RHS (12 point sources at site 0 + 4 Gaussian, each through M^dag) in one
    batched FP16 solve: every RHS converges.

At these sizes the numpy oracle takes minutes per application, so the checks
are size-independent properties: the residual of the returned x recomputed
with the reference-layout FP64 operator (a kernel separate from the solver's),
and the distance between the mixed and the plain FP64 solutions, which two
solutions with true residual <= 1e-10 can differ by at most
cond(M^dag M) * 2e-10 (cond < 1e4 here), so 2e-6 relative is the bound.
"""

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("CUDA device required", allow_module_level=True)

from jaxqft_b200.lib import SLOT_CONVERGED, WilsonContext  # noqa: E402

BC = (1, 1, 1, -1)


def _links(shape, scale, seed, dev):
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    shp = (4, *shape, 3, 3)
    a = scale * torch.complex(torch.randn(shp, generator=g, device=dev, dtype=torch.float64),
                              torch.randn(shp, generator=g, device=dev, dtype=torch.float64))
    y = 0.5 * (a - a.conj().transpose(-1, -2))
    del a
    tr = torch.diagonal(y, dim1=-2, dim2=-1).sum(-1) / 3.0
    y = y - tr[..., None, None] * torch.eye(3, dtype=y.dtype, device=dev)
    return torch.linalg.matrix_exp(y)


def _even_mask(shape, dev):
    x = [torch.arange(n, device=dev) for n in shape]
    par = (x[0][:, None, None, None] + x[1][None, :, None, None] + x[2][None, None, :, None]
           + x[3][None, None, None, :]) % 2
    return (par == 0).to(torch.complex128)[..., None, None]


def _gauss(n, shape, seed, dev):
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    shp = (n, *shape, 4, 3)
    return torch.complex(torch.randn(shp, generator=g, device=dev, dtype=torch.float64),
                         torch.randn(shp, generator=g, device=dev, dtype=torch.float64)) / math.sqrt(2.0)


def _true_res(ctx, gauge, mass, x, b):
    Ax = ctx.apply("SCHUR_E_NORMAL", gauge, mass, x, normalized=True)
    r = (b - Ax).reshape(b.shape[0], -1)
    return (torch.linalg.vector_norm(r, dim=1) / torch.linalg.vector_norm(b.reshape(b.shape[0], -1), dim=1)).cpu()


@pytest.fixture(scope="module")
def c2():
    dev = torch.device("cuda", 0)
    shape = (16, 16, 16, 32)
    kappa = 0.135
    mass = 1.0 / (2.0 * kappa) - 4.0
    ctx = WilsonContext(shape, bc=BC, device=dev)
    gauge = ctx.gauge(_links(shape, 0.2, 11, dev))
    eta = _gauss(1, shape, 12, dev) * _even_mask(shape, dev)
    b = ctx.apply("SCHUR_E_DAG", gauge, mass, eta, normalized=True)
    x64, st64 = ctx.solve(gauge, b, mass, op="eo_normal", tol=1e-10, maxiter=4000, inner="double")
    assert st64[0]["status"] == SLOT_CONVERGED
    return ctx, gauge, mass, b, x64, st64


@pytest.mark.parametrize("inner", ["single", "half"])
def test_c2_mixed_eo_solve_matches_fp64(c2, inner):
    ctx, gauge, mass, b, x64, st64 = c2
    x, st = ctx.solve(gauge, b, mass, op="eo_normal", tol=1e-10, maxiter=4000, inner=inner)
    assert st[0]["status"] == SLOT_CONVERGED, st
    assert st[0]["true_res"] <= 1e-10
    assert float(_true_res(ctx, gauge, mass, x, b)[0]) <= 1.05e-10
    d = float(torch.linalg.vector_norm(x - x64) / torch.linalg.vector_norm(x64))
    assert d <= 2e-6, d
    # the mixed solve needs at most a few percent more iterations than FP64 CG
    assert st[0]["iters"] <= 1.2 * st64[0]["iters"] + 10, (st, st64)


def test_c3_batched_half_kappa_0130_full_size():
    dev = torch.device("cuda", 0)
    shape = (24, 24, 24, 48)
    kappa = 0.130
    mass = 1.0 / (2.0 * kappa) - 4.0
    ctx = WilsonContext(shape, bc=BC, device=dev)
    gauge = ctx.gauge(_links(shape, 0.2, 0, dev))
    eta = torch.zeros((16, *shape, 4, 3), dtype=torch.complex128, device=dev)
    for k in range(12):
        eta[k, 0, 0, 0, 0, k // 3, k % 3] = 1.0
    eta[12:] = _gauss(4, shape, 5, dev)
    b = ctx.apply("SCHUR_E_DAG", gauge, mass, eta * _even_mask(shape, dev), normalized=True)
    del eta
    x, st = ctx.solve(gauge, b, mass, op="eo_normal", tol=1e-10, maxiter=4000, inner="half")
    assert all(s["status"] == SLOT_CONVERGED for s in st), st
    res = _true_res(ctx, gauge, mass, x, b).numpy()
    assert np.all(res <= 1.05e-10), res
    reported = np.array([s["true_res"] for s in st])
    assert np.allclose(res, reported, rtol=0.05, atol=1e-13), (res, reported)
