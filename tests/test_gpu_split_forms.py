"""Split solver forms against the normal form, following the reference's own
consistency check ``test_pseudofermion_solver_consistency``
(jaxqft/models/su3_wilson_nf2.py:2303-2412): for phi from a heatbath refresh,

* normal: x_n = (A^dag A)^-1 phi, residual A^dag A x_n - phi;
* split: y = A^-dag phi, x = A^-1 y with stage residuals A^dag y - phi, A x - y, the
  total residual A^dag A x - phi, x against x_n and S = y^dag y against phi^dag x_n;
* eo_split (unpreconditioned monomial): the same pair through the even Schur complement
  (solve_dagger_eo / solve_direct_eo, :1301-1336).

The reference runs these with BiCGStab; the B200 theory serves every non-Hermitian
solve with CG on the normal equations, so the bar is the same set of identities at
the solver tolerance.  cg_tol = 1e-11 on the normal residual; the stage residuals
carry one condition-number factor of D (~10 at mass -0.2 on these links), hence
the 1e-8 bounds.
"""

import numpy as np
import pytest

from oracle import wilson as W

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("CUDA device required", allow_module_level=True)

from jaxqft_b200.su3_wilson_nf2 import SU3WilsonNf2  # noqa: E402

SHAPE = (4, 4, 4, 8)
BC = (1, 1, 1, -1)


def _theory(kind, form, kind_solver="bicgstab", **kw):
    return SU3WilsonNf2(lattice_shape=SHAPE, beta=5.6, mass=-0.2, fermion_bc=BC, cg_tol=1e-11, cg_maxiter=5000,
                        fermion_monomial_kind=kind, solver_kind=kind_solver, solver_form=form,
                        pseudofermion_force_mode="analytic", solver_precision="single", batch_size=2, seed=7, **kw)


def _links(seed, scale=0.3, batch=2):
    return torch.from_numpy(W.hot_links(np.random.default_rng(seed), SHAPE, batch, scale)).cuda()


def _rel(a, b):
    a, b = a.reshape(a.shape[0], -1), b.reshape(b.shape[0], -1)
    return float((torch.linalg.vector_norm(a, dim=1) / torch.linalg.vector_norm(b, dim=1)).max())


def test_split_requires_non_hermitian_kind():
    with pytest.raises(ValueError, match="non-Hermitian"):
        _theory("unpreconditioned", "split", kind_solver="cg")
    with pytest.raises(ValueError, match="solver_form"):
        _theory("unpreconditioned", "lu")


def test_unpreconditioned_split_and_eo_split():
    th = _theory("unpreconditioned", "split")
    U = _links(1)
    m = th.fermion_monomial
    m.refresh(U)
    phi = m.phi
    x_n = th.solve_normal(U, phi)
    assert _rel(th.apply_normal(U, x_n) - phi, phi) < 1e-10
    x_s, y_s = th.solve_split_with_intermediate(U, phi)
    assert _rel(th.apply_Ddag(U, y_s) - phi, phi) < 1e-8
    assert _rel(th.apply_D(U, x_s) - y_s, y_s) < 1e-8
    assert _rel(th.apply_normal(U, x_s) - phi, phi) < 1e-10
    assert _rel(x_s - x_n, x_n) < 1e-8
    Sn = torch.stack([(phi[b].conj() * x_n[b]).sum().real for b in range(2)])
    Ss = torch.stack([(y_s[b].conj() * y_s[b]).sum().real for b in range(2)])
    assert float(((Sn - Ss).abs() / Sn.abs()).max()) < 1e-9
    # eo pair through the Schur complement
    y_e = th.solve_dagger_eo(U, phi)
    x_e = th.solve_direct_eo(U, y_e)
    assert _rel(th.apply_Ddag(U, y_e) - phi, phi) < 1e-8
    assert _rel(th.apply_D(U, x_e) - y_e, y_e) < 1e-8
    assert _rel(x_e - x_n, x_n) < 1e-8
    # single direct / dagger solves
    b = th.random_fermion()
    assert _rel(th.apply_D(U, th.solve_direct(U, b)) - b, b) < 1e-8
    assert _rel(th.apply_Ddag(U, th.solve_dagger(U, b)) - b, b) < 1e-8
    # the monomial action in split form: S = chi^dag chi = eta^dag eta after a heatbath refresh
    spf = m.action(U)
    eta2 = torch.stack([(m.eta[b].conj() * m.eta[b]).sum().real for b in range(2)])
    assert float(((spf - eta2).abs() / eta2).max()) < 1e-9


def test_eo_split_form_monomial_matches_normal():
    U = _links(2)
    th_n = _theory("unpreconditioned", "normal", kind_solver="cg")
    th_s = _theory("unpreconditioned", "eo_split")
    th_n.prepare_trajectory(U)
    th_s.set_loaded_pseudofermion(th_n.fermion_monomial.phi)
    sn, ss = th_n.fermion_monomial.action(U), th_s.fermion_monomial.action(U)
    assert float(((sn - ss).abs() / sn.abs()).max()) < 1e-9
    Fn = th_n.fermion_monomial.force(U)
    Fs = th_s.fermion_monomial.force(U)
    assert _rel(Fs - Fn, Fn) < 1e-8


def test_eo_preconditioned_split():
    th = _theory("eo_preconditioned", "split")
    U = _links(3)
    m = th.fermion_monomial
    m.refresh(U)
    phi = m.phi
    x_n = th.solve_eop_even_normal(U, phi)
    x_s, y_s = th.solve_eop_even_split_with_intermediate(U, phi)
    r1 = th.apply_eo_schur_even_dagger(U, y_s, normalized=True) - phi
    r2 = th.apply_eo_schur_even(U, x_s, normalized=True) - y_s
    assert _rel(r1, phi) < 1e-8 and _rel(r2, y_s) < 1e-8
    assert _rel(x_s - x_n, x_n) < 1e-8
    spf = m.action(U)
    eta2 = torch.stack([(m.eta[b].conj() * m.eta[b]).sum().real for b in range(2)])
    assert float(((spf - eta2).abs() / eta2).max()) < 1e-9
    # direct / dagger Schur solves
    b = th._project_even(th.random_fermion())
    assert _rel(th.apply_eo_schur_even(U, th.solve_eop_even_direct(U, b), normalized=True) - b, b) < 1e-8
    assert _rel(th.apply_eo_schur_even_dagger(U, th.solve_eop_even_dagger(U, b), normalized=True) - b, b) < 1e-8
    # split-form force equals the normal-form force
    th_n = _theory("eo_preconditioned", "normal", kind_solver="cg")
    th_n.set_loaded_pseudofermion(phi)
    assert _rel(m.force(U) - th_n.fermion_monomial.force(U), th_n.fermion_monomial.force(U)) < 1e-8


@pytest.mark.parametrize("kind", ["unpreconditioned", "eo_preconditioned"])
def test_split_form_hmc_chain_matches_normal(kind):
    """Two MinNorm2 trajectories with the same momenta, pseudofermion noise and uniforms:
    the split-form theory reproduces the normal-form dH and the final links."""
    from jaxqft_b200.integrators import MinNorm2
    from jaxqft_b200.update import HMC

    rng = np.random.default_rng(11)
    U0 = W.hot_links(rng, SHAPE, 1, 0.1)
    Ps = [W.algebra_field(rng, SHAPE, 1) for _ in range(2)]
    etas = [W.gaussian_spinor(rng, SHAPE, 1) for _ in range(2)]
    Rs = [0.5, 0.5]
    runs = []
    for form, ks in (("normal", "cg"), ("split", "bicgstab")):
        th = SU3WilsonNf2(lattice_shape=SHAPE, beta=5.6, mass=0.1, fermion_bc=BC, cg_tol=1e-12, cg_maxiter=5000,
                          fermion_monomial_kind=kind, solver_kind=ks, solver_form=form, solver_precision="single")
        it_P, it_eta, it_R = iter(Ps), iter(etas), iter(Rs)
        th.refreshP = lambda it=it_P: torch.from_numpy(next(it)).cuda()
        th.random_fermion = lambda it=it_eta: torch.from_numpy(next(it)).cuda()
        hmc = HMC(th, MinNorm2(th.force, th.evolve_q, 4, 0.5), verbose=False, uniform=lambda shp, it=it_R: [next(it)])
        U = hmc.evolve(torch.from_numpy(U0).cuda(), 2)
        runs.append(([h["dH"][0] for h in hmc.history], U.cpu().numpy()))
    (dh_n, U_n), (dh_s, U_s) = runs
    for a, b in zip(dh_n, dh_s):
        assert abs(a - b) < 1e-7 * max(1.0, abs(a)), (dh_n, dh_s)
    assert np.linalg.norm(U_s - U_n) / np.linalg.norm(U_n) < 1e-9
