"""Every non-Hermitian solve form meets the reference's own stopping rule.

The reference solves A x = b with BiCGStab / GMRES (jax.scipy.sparse.linalg,
tol relative, atol 0; jaxqft/models/su3_wilson_nf2.py:1217-1299, 1301-1364),
so its solutions satisfy ||b - A x|| <= cg_tol ||b|| for A = D, D^dag, the
unnormalized even Schur operator S_e (solve_direct_eo / solve_dagger_eo), and
the normalized one M, M^dag (solve_eop_even_direct / _dagger).  The B200 theory
serves them with CG on the normal equations plus FP64 defect correction; here
the residual of each returned solution is recomputed with the FP64 operators
at kappa 0.135 (bare mass -0.2963) and must meet the rule, for FP64 and for
FP32 / FP16 inner iterations, with the split forms' stage residuals too.
"""

import numpy as np
import pytest

from oracle import wilson as W

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("CUDA device required", allow_module_level=True)

from jaxqft_b200.su3_wilson_nf2 import SU3WilsonNf2  # noqa: E402

SHAPE = (8, 8, 8, 16)
BC = (1, 1, 1, -1)
MASS = W.kappa_to_mass(0.135)


def _rel(r, b):
    r, b = r.reshape(r.shape[0], -1), b.reshape(b.shape[0], -1)
    return (torch.linalg.vector_norm(r, dim=1) / torch.linalg.vector_norm(b, dim=1)).cpu().numpy()


@pytest.fixture(scope="module")
def fields():
    rng = np.random.default_rng(21)
    U = torch.from_numpy(W.hot_links(rng, SHAPE, 2, 0.2)).cuda()
    b = torch.from_numpy(W.gaussian_spinor(rng, SHAPE, 2)).cuda()
    return U, b


@pytest.mark.parametrize("precision", ["double", "single", "half"])
@pytest.mark.parametrize("tol", [1e-8, 1e-10])
def test_direct_and_dagger_forms_meet_reference_rule(fields, precision, tol):
    U, b = fields
    th = SU3WilsonNf2(lattice_shape=SHAPE, beta=5.6, mass=MASS, fermion_bc=BC, cg_tol=tol, cg_maxiter=20000,
                      solver_kind="bicgstab", solver_precision=precision, batch_size=2)
    m0 = MASS + 4.0
    be, bo = th._project_even(b), th._project_odd(b)

    x = th.solve_direct(U, b)
    assert (_rel(b - th.apply_D(U, x), b) <= tol).all()
    y = th.solve_dagger(U, b)
    assert (_rel(b - th.apply_Ddag(U, y), b) <= tol).all()

    # EO forms: the Schur system S_e x_e = b_e - P_e K b_o / m0 (unnormalized, K = D - m0), then
    # x_o = (b_o - P_o K x_e) / m0; the reference's stopping rule is on the Schur system
    for name, op, fn in (("direct", th.apply_D, th.solve_direct_eo), ("dagger", th.apply_Ddag, th.solve_dagger_eo)):
        x = fn(U, b)
        K = lambda v: op(U, v) - m0 * v  # noqa: E731
        rhs_e = be - th._project_even(K(bo)) / m0
        xe = th._project_even(x)
        Se = m0 * xe - th._project_even(K(th._project_odd(K(xe)))) / m0
        assert (_rel(rhs_e - Se, rhs_e) <= tol).all(), name
        # the odd reconstruction makes the full system exact up to that residual
        assert (_rel(b - op(U, x), b) <= 10 * tol).all(), name

    x = th.solve_eop_even_direct(U, be)
    assert (_rel(be - th.apply_eo_schur_even(U, x, normalized=True), be) <= tol).all()
    y = th.solve_eop_even_dagger(U, be)
    assert (_rel(be - th.apply_eo_schur_even_dagger(U, y, normalized=True), be) <= tol).all()


@pytest.mark.parametrize("form", ["split", "eo_split"])
def test_split_stages_meet_reference_rule(fields, form):
    U, b = fields
    tol = 1e-9
    th = SU3WilsonNf2(lattice_shape=SHAPE, beta=5.6, mass=MASS, fermion_bc=BC, cg_tol=tol, cg_maxiter=20000,
                      solver_kind="bicgstab", solver_form=form, solver_precision="single", batch_size=2)
    x, y = th.solve_split_with_intermediate(U, b)
    assert (_rel(b - th.apply_Ddag(U, y), b) <= (tol if form == "split" else 10 * tol)).all()
    assert (_rel(y - th.apply_D(U, x), y) <= (tol if form == "split" else 10 * tol)).all()
    x2, y2 = th.solve_eop_even_split_with_intermediate(U, th._project_even(b))
    be = th._project_even(b)
    assert (_rel(be - th.apply_eo_schur_even_dagger(U, y2, normalized=True), be) <= tol).all()
    assert (_rel(y2 - th.apply_eo_schur_even(U, x2, normalized=True), y2) <= tol).all()
