"""The reference's own known-answer identities for the Wilson Nf=2 path
(jaxqft/models/su3_wilson_nf2.py), run on the GPU through the drop-in theory:

* pseudofermion refresh identity (2085-2116): after a heatbath refresh
  phi = D^dag eta (or phi_e = S_e^dag eta_e), S_pf = phi^dag (A)^-1 phi = eta^dag eta;
* force against the central finite difference of the action along a random
  algebra direction H (2472-2599, eps = 5e-4): (S(e^{eps H} U) - S(e^{-eps H} U)) / (2 eps)
  = -<F, H> with <a, b> = -Re Tr(a b) summed over links;
* gauge covariance (1988-2037, 1674-1676): with U'_mu(x) = W(x)^dag U_mu(x) W(x+mu) and
  psi' = W^dag psi, D[U'] psi' = W^dag D[U] psi, and the actions are gauge invariant.
"""

import numpy as np
import pytest

from oracle import wilson as W

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("CUDA device required", allow_module_level=True)

from jaxqft_b200.su3_wilson_nf2 import SU3WilsonNf2  # noqa: E402

SHAPE = (4, 4, 4, 6)
BC = (1, 1, 1, -1)


def _theory(kind, **kw):
    return SU3WilsonNf2(lattice_shape=SHAPE, beta=5.6, mass=-0.2, fermion_bc=BC, cg_tol=1e-11, cg_maxiter=5000,
                        action_cg_tol=1e-12, fermion_monomial_kind=kind, pseudofermion_force_mode="analytic",
                        solver_precision="single", seed=5, **kw)


def _links(seed, scale=0.3):
    return torch.from_numpy(W.hot_links(np.random.default_rng(seed), SHAPE, 1, scale)).cuda()


@pytest.mark.parametrize("kind", ["unpreconditioned", "eo_preconditioned"])
def test_refresh_identity(kind):
    th = _theory(kind)
    U = _links(1)
    th.prepare_trajectory(U)
    m = th.fermion_monomial
    spf = float(m.action(U)[0])
    eta2 = float((m.eta.conj() * m.eta).real.sum())
    assert abs(spf - eta2) / eta2 < 1e-9, (spf, eta2)


@pytest.mark.parametrize("kind", ["unpreconditioned", "eo_preconditioned"])
def test_force_matches_central_difference(kind):
    th = _theory(kind)
    U = _links(2)
    th.prepare_trajectory(U)
    eps = 5e-4
    H = torch.from_numpy(W.algebra_field(np.random.default_rng(3), SHAPE, 1)).cuda()
    Sp = float(th.action(th.evolve_q(eps, H, U))[0])
    Sm = float(th.action(th.evolve_q(-eps, H, U))[0])
    fd = (Sp - Sm) / (2.0 * eps)
    F = th.force(U)
    directional = float(torch.einsum("...ab,...ba->...", F, H).real.sum())  # -<F, H>
    assert abs(fd - directional) <= 1e-5 * abs(directional), (fd, directional)


def _random_su3(rng, n):
    return W.hot_links(rng, (1, 1, 1, n), 1, 1.0)[0, 0, 0, 0, 0]  # n SU(3) matrices [n][3][3]


def test_gauge_covariance():
    th = _theory("unpreconditioned")
    rng = np.random.default_rng(4)
    U = W.hot_links(rng, SHAPE, 1, 0.3)
    V = int(np.prod(SHAPE))
    Om = _random_su3(rng, V).reshape(*SHAPE, 3, 3)
    Od = np.conj(np.swapaxes(Om, -1, -2))
    Up = np.empty_like(U)
    for mu in range(4):
        Om_fwd = np.roll(Om, -1, axis=mu)  # Omega(x + mu)
        Up[0, mu] = Od @ U[0, mu] @ Om_fwd
    psi = W.gaussian_spinor(rng, SHAPE, 1)
    psip = np.einsum("...ab,n...sb->n...sa", Od, psi)
    Dpsi = th.apply_D(torch.from_numpy(U).cuda(), torch.from_numpy(psi).cuda()).cpu().numpy()
    Dpsip = th.apply_D(torch.from_numpy(Up).cuda(), torch.from_numpy(psip).cuda()).cpu().numpy()
    expect = np.einsum("...ab,n...sb->n...sa", Od, Dpsi)
    assert np.linalg.norm(Dpsip - expect) / np.linalg.norm(expect) < 1e-13
    # gauge action and the pseudofermion action (phi transformed with the links) are invariant
    Ut, Upt = torch.from_numpy(U).cuda(), torch.from_numpy(Up).cuda()
    assert abs(float(th.gauge_action(Ut)[0]) - float(th.gauge_action(Upt)[0])) < 1e-10 * abs(float(th.gauge_action(Ut)[0]))
    phi = th.apply_Ddag(Ut, torch.from_numpy(psi).cuda())
    phip = torch.from_numpy(np.einsum("...ab,n...sb->n...sa", Od, phi.cpu().numpy())).cuda()
    th.set_loaded_pseudofermion(phi)
    s0 = float(th.fermion_monomial.action(Ut)[0])
    th.set_loaded_pseudofermion(phip)
    s1 = float(th.fermion_monomial.action(Upt)[0])
    assert abs(s0 - s1) < 1e-9 * abs(s0), (s0, s1)


@pytest.mark.parametrize("kind", ["unpreconditioned", "eo_preconditioned"])
def test_force_gauge_covariance(kind):
    """Pseudofermion force covariance (su3_wilson_nf2.py:2415-2469): with
    U'_mu(x) = Om(x)^dag U_mu(x) Om(x+mu) and phi' = Om^dag phi, the analytic
    force satisfies F_mu[U', phi'](x) = Om(x)^dag F_mu[U, phi](x) Om(x)."""
    th = _theory(kind)
    rng = np.random.default_rng(6)
    U = W.hot_links(rng, SHAPE, 1, 0.3)
    V = int(np.prod(SHAPE))
    Om = _random_su3(rng, V).reshape(*SHAPE, 3, 3)
    Od = np.conj(np.swapaxes(Om, -1, -2))
    Up = np.empty_like(U)
    for mu in range(4):
        Up[0, mu] = Od @ U[0, mu] @ np.roll(Om, -1, axis=mu)
    Ut = torch.from_numpy(U).cuda()
    m = th.fermion_monomial
    m.refresh(Ut)
    phi = m.phi.cpu().numpy()
    phip = np.einsum("...ab,n...sb->n...sa", Od, phi)  # site-local: odd sites of an even phi stay zero
    F = m.force_analytic(Ut, torch.from_numpy(phi).cuda()).cpu().numpy()
    Fp = m.force_analytic(torch.from_numpy(Up).cuda(), torch.from_numpy(phip).cuda()).cpu().numpy()
    Fcov = np.stack([Od @ F[:, mu] @ Om for mu in range(4)], axis=1)
    assert np.linalg.norm(Fp - Fcov) / np.linalg.norm(Fcov) < 1e-8
