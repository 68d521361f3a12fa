"""Point-source propagator and pion two-point function on the GPU against the
reference's own measurement code (golden_meas.npz: jaxqft/core/measurements.py
277-390 run on 4^4 with an odd-parity source) and against the oracle.

Tolerances: propagators 1e-9 relative (both sides solve to a true residual of
1e-12 on D^dag D, cond < 1e3 at this kappa); the contraction kernel alone is
FP64 summation, 1e-13."""

import numpy as np
import pytest

from oracle import wilson as W
from tests.conftest import load_golden, rel

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("CUDA device required", allow_module_level=True)

from jaxqft_b200 import measurements as M  # noqa: E402
from jaxqft_b200.lib import WilsonContext  # noqa: E402
from jaxqft_b200.su3_wilson_nf2 import SU3WilsonNf2  # noqa: E402


@pytest.fixture(scope="module")
def golden():
    return load_golden("meas")


@pytest.mark.parametrize("method", ["normal", "eo"])
@pytest.mark.parametrize("prec", ["double", "single"])
def test_propagator_and_pion_match_reference(golden, method, prec):
    g = golden
    th = SU3WilsonNf2(lattice_shape=tuple(int(v) for v in g["shape"]), beta=5.6, mass=float(g["mass"]),
                      fermion_bc=(1, 1, 1, -1), cg_tol=1e-12, cg_maxiter=5000, solver_precision=prec)
    U = torch.from_numpy(g["U"]).cuda()
    prop, info = M.point_source_propagator(th, U, tuple(int(v) for v in g["source"]), method=method)
    assert info["inv_all_converged"] == 1.0 and info["inv_n_solves"] == 12
    assert rel(prop.cpu().numpy(), g["prop"]) < 1e-9
    corr = M.pion_two_point(th.ctx, prop, int(g["source"][3]))
    assert np.allclose(corr, g["pion"], rtol=1e-9, atol=0)


def test_pion_kernel_against_oracle():
    shape = (8, 4, 6, 12)
    rng = np.random.default_rng(3)
    cols = (rng.standard_normal((12, *shape, 4, 3)) + 1j * rng.standard_normal((12, *shape, 4, 3)))
    ctx = WilsonContext(shape, bc=(1, 1, 1, -1))
    prop = np.moveaxis(cols.reshape(4, 3, *shape, 4, 3), (0, 1), (-2, -1))[None]  # (1, *L, s, c, s0, c0)
    for t0 in (0, 5, 11):
        ref = W.pion_two_point(prop, t0)
        assert np.allclose(ctx.pion_correlator(torch.from_numpy(cols), t0), ref, rtol=1e-13, atol=0)
        assert np.allclose(M.pion_two_point(ctx, torch.from_numpy(prop).cuda(), t0), ref, rtol=1e-13, atol=0)
