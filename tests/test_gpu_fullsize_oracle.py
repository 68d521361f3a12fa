"""Full-size operator applications against an independent CPU oracle.

At 16^3x32 and 24^3x48 (the lattices of the measured configurations) the
numpy oracle is too slow, so the checker is the C restatement of the
reference's compact hops (oracle/c/wilson_cpu.c, itself pinned to the numpy
oracle in tests/test_oracle_c.py): D and D^dag on the reference layout
(wl_apply, the drop-in path), and the normalized even Schur normal operator
M^dag M that solve_eop_even_normal inverts (wl_apply SCHUR_E_NORMAL), all in
FP64 at 1e-13 relative, on seeded links exp(i*0.2*H) and Gaussian spinors.
References: jaxqft/fermions/wilson.py:171-284, models/su3_wilson_nf2.py:976-988.
"""

import math

import numpy as np
import pytest

from oracle import cpu as C
from oracle import wilson as W
from tests.conftest import rel

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("CUDA device required", allow_module_level=True)

from jaxqft_b200.lib import WilsonContext  # noqa: E402

BC = (1, 1, 1, -1)
TOL = 1e-13


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


def _gauss(shape, seed, dev):
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    shp = (1, *shape, 4, 3)
    return torch.complex(torch.randn(shp, generator=g, device=dev, dtype=torch.float64),
                         torch.randn(shp, generator=g, device=dev, dtype=torch.float64)) / math.sqrt(2.0)


@pytest.mark.parametrize("shape,kappa", [((16, 16, 16, 32), 0.135), ((24, 24, 24, 48), 0.135),
                                         ((24, 24, 24, 48), 0.130)])
def test_fullsize_operators_match_c_oracle(shape, kappa):
    dev = torch.device("cuda", 0)
    mass = 1.0 / (2.0 * kappa) - 4.0
    ctx = WilsonContext(shape, bc=BC, device=dev)
    U = _links(shape, 0.2, 41, dev)
    gauge = ctx.gauge(U)
    psi = _gauss(shape, 42, dev)
    D = ctx.apply("D", gauge, mass, psi).cpu().numpy()[0]
    Dd = ctx.apply("DDAG", gauge, mass, psi).cpu().numpy()[0]
    xe = psi * torch.from_numpy(W.mask(shape, 0)).to(dev)
    N = ctx.apply("SCHUR_E_NORMAL", gauge, mass, xe, normalized=True).cpu().numpy()
    del xe
    torch.cuda.synchronize()
    C.build()
    cw = C.CpuWilson(U.cpu().numpy(), shape, BC, mass)
    del U
    p = psi.cpu().numpy()
    assert rel(D, cw.apply_D(p[0])) < TOL
    assert rel(Dd, cw.apply_D(p[0], dag=True)) < TOL
    ref = cw.normal(W.pack(p, 0)[0])
    assert rel(W.pack(N, 0)[0], ref) < TOL
    assert np.abs(W.pack(N, 1)).max() == 0.0  # odd sites of the Schur result are zero
