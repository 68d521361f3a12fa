"""The device random fields (wl_random_spinor, wl_random_algebra): equal to the
numpy restatement oracle/rng.py on a small lattice (Philox4x32-10 words are
exact; the Box-Muller log / sqrt / sincospi of CUDA and numpy differ by a few
ulps, hence 1e-13), and with the moments the reference's draws have
(random_fermion, jaxqft/models/su3_wilson_nf2.py:1169-1175: complex Gaussian,
E z = 0, E|z|^2 = 1, E|z|^4 = 2; _sample_algebra, jaxqft/models/su3_ym.py:
238-244: anti-Hermitian, traceless, E|P_ab|^2 = scale^2 off the diagonal and
2/3 scale^2 on it) at 16^3x32, each to five standard errors."""

import numpy as np
import pytest

from oracle import rng as R

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("CUDA device required", allow_module_level=True)

from jaxqft_b200.lib import WilsonContext  # noqa: E402


def test_fields_match_numpy_restatement():
    shape = (4, 4, 4, 4)
    V = 256
    ctx = WilsonContext(shape)
    seed, stream = (1 << 40) + 12345, (7 << 33) + 3
    z = ctx.random_spinor(2, seed, stream).cpu().numpy().reshape(2, V, 4, 3)
    np.testing.assert_allclose(z, R.random_spinor(seed, stream, 2, V), rtol=0, atol=1e-13)
    P = ctx.random_algebra(2, seed, stream, scale=0.3).cpu().numpy().reshape(2, 4 * V, 3, 3)
    np.testing.assert_allclose(P, R.random_algebra(seed, stream, 2, V, 0.3), rtol=0, atol=1e-13)


def test_same_seed_and_stream_repeat_and_others_differ():
    ctx = WilsonContext((4, 4, 4, 8))
    a = ctx.random_spinor(1, 5, 1)
    assert torch.equal(a, ctx.random_spinor(1, 5, 1))
    assert not torch.allclose(a, ctx.random_spinor(1, 5, 2))
    assert not torch.allclose(a, ctx.random_spinor(1, 6, 1))
    two = ctx.random_spinor(2, 5, 1)
    assert torch.equal(two[0], a[0]) and not torch.allclose(two[1], a[0])  # fields of one call differ


def test_spinor_moments():
    ctx = WilsonContext((16, 16, 16, 32))
    z = ctx.random_spinor(2, 11, 1).reshape(-1)
    n = z.numel()
    for part in (z.real, z.imag):  # each N(0, 1/2)
        assert abs(float(part.mean())) < 5 * (0.5 / n) ** 0.5
    a2 = (z.abs() ** 2)
    assert abs(float(a2.mean()) - 1.0) < 5 * (1.0 / n) ** 0.5          # Var|z|^2 = 1
    assert abs(float((a2 ** 2).mean()) - 2.0) < 5 * (20.0 / n) ** 0.5  # Var|z|^4 = E|z|^8 - 4 = 20
    c = (z[:-1] * z[1:].conj()).mean()  # neighbouring components uncorrelated
    assert abs(complex(c)) < 5 * (1.0 / n) ** 0.5


@pytest.mark.parametrize("scale", [1.0, 0.2])
def test_algebra_moments(scale):
    ctx = WilsonContext((16, 16, 16, 32))
    P = ctx.random_algebra(1, 3, 9, scale=scale).reshape(-1, 3, 3)
    assert float((P + P.conj().transpose(-1, -2)).abs().max()) == 0.0
    assert float(torch.diagonal(P, dim1=-2, dim2=-1).sum(-1).abs().max()) < 1e-15 * scale * 10
    off = torch.cat([P[:, 0, 1], P[:, 0, 2], P[:, 1, 2]]).abs() ** 2 / scale ** 2
    dia = torch.diagonal(P, dim1=-2, dim2=-1).reshape(-1).abs() ** 2 / scale ** 2
    assert abs(float(off.mean()) - 1.0) < 5 * (1.0 / off.numel()) ** 0.5
    # diagonal: i (h_a - mean h), h ~ N(0, 1): E = 2/3, Var = 2 (2/3)^2; entries of a link are correlated
    assert abs(float(dia.mean()) - 2.0 / 3.0) < 5 * (3 * 2 * (2 / 3) ** 2 / dia.numel()) ** 0.5
