"""Gauge-sector kernels (plaquette sum, staple force, exp(dt P) U drift,
kinetic term) through the C-ABI against the numpy oracle, which follows
jaxqft/models/su3_ym.py (plaquette 274-286, staple force 298-327, drift with
expm 349-350, kinetic 362-364).  FP64 throughout; tolerance 1e-13 relative
(observed ~1e-15).  The reference's own outputs for these pieces are checked
through the theory mirror in test_gpu_theory.py."""

import numpy as np
import pytest

from oracle import wilson as W
from tests.conftest import rel

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("CUDA device required", allow_module_level=True)

from jaxqft_b200.lib import WilsonContext  # noqa: E402
from jaxqft_b200.su3_ym import SU3YangMills  # noqa: E402

SHAPE = (6, 4, 4, 8)


@pytest.fixture(scope="module")
def fields():
    rng = np.random.default_rng(21)
    U = W.hot_links(rng, SHAPE, 2, 0.5)
    P = W.algebra_field(rng, SHAPE, 2)
    ctx = WilsonContext(SHAPE, bc=(1, 1, 1, 1))
    return ctx, U, P


def test_plaquette_sum_and_kinetic(fields):
    ctx, U, P = fields
    assert np.allclose(ctx.plaquette_sum(torch.from_numpy(U)), W.plaquette_sum(U), rtol=1e-13, atol=0)
    assert np.allclose(ctx.kinetic(torch.from_numpy(P)), W.kinetic(P), rtol=1e-13, atol=0)


def test_staple_force(fields):
    ctx, U, _ = fields
    F = ctx.gauge_force(torch.from_numpy(U), 5.6).cpu().numpy()
    ref = W.gauge_force(U, 5.6)
    assert rel(F, ref) < 1e-13
    # traceless anti-Hermitian per link
    assert np.abs(F + np.conj(np.swapaxes(F, -1, -2))).max() < 1e-14
    assert np.abs(np.trace(F, axis1=-2, axis2=-1)).max() < 1e-14


@pytest.mark.parametrize("dt", [0.1, 0.7, 3.0])
def test_exponential_drift(fields, dt):
    """dt up to 3 makes ||dt P|| > 1/2 so the scaling-and-squaring steps run."""
    ctx, U, P = fields
    out = ctx.gauge_evolve(dt, torch.from_numpy(P), torch.from_numpy(U)).cpu().numpy()
    assert rel(out, W.evolve_q(dt, P, U)) < 1e-13
    eye = np.eye(3)
    assert np.abs(out @ np.conj(np.swapaxes(out, -1, -2)) - eye).max() < 1e-13
    assert np.abs(np.linalg.det(out) - 1.0).max() < 1e-13


def test_drift_in_place(fields):
    ctx, U, P = fields
    Ut = torch.from_numpy(U).cuda().clone()
    ctx.gauge_evolve(0.2, torch.from_numpy(P), Ut, out=Ut)
    assert rel(Ut.cpu().numpy(), W.evolve_q(0.2, P, U)) < 1e-13


@pytest.mark.parametrize("layout", ["BMXYIJ", "BXYMIJ"])
def test_theory_mirror_layouts(fields, layout):
    _, U, P = fields
    th = SU3YangMills(SHAPE, beta=5.6, batch_size=2, layout=layout)
    Ut, Pt = torch.from_numpy(U).cuda(), torch.from_numpy(P).cuda()
    if layout == "BXYMIJ":
        Ut, Pt = Ut.movedim(1, 5), Pt.movedim(1, 5)
    assert np.allclose(th.action(Ut).cpu().numpy(), W.gauge_action(U, 5.6), rtol=1e-13)
    F = th.force(Ut)
    U2 = th.evolve_q(0.3, Pt, Ut)
    if layout == "BXYMIJ":
        F, U2 = F.movedim(5, 1), U2.movedim(5, 1)
    assert rel(F.cpu().numpy(), W.gauge_force(U, 5.6)) < 1e-13
    assert rel(U2.cpu().numpy(), W.evolve_q(0.3, P, U)) < 1e-13
    assert np.allclose(th.kinetic(Pt).cpu().numpy(), W.kinetic(P), rtol=1e-13)


def test_lime_configuration_on_device():
    """A SciDAC LIME configuration read straight into device memory feeds the
    gauge kernels: plaquette of the file = oracle plaquette of the stored links."""
    import os

    from jaxqft_b200 import lime
    from tests.conftest import GOLDEN, load_golden

    g = load_golden("lime")
    U = lime.load_gauge(os.path.join(GOLDEN, "gauge_D.lime"))
    assert U.is_cuda and U.dtype == torch.complex128
    shape = tuple(U.shape[2:6])
    ctx = WilsonContext(shape, bc=(1, 1, 1, 1))
    assert np.allclose(ctx.plaquette_sum(U), W.plaquette_sum(g["U_D"]), rtol=1e-13, atol=0)
