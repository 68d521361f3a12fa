"""HMC chain parity: the GPU HMC (jaxqft_b200.update.HMC driving SU3WilsonNf2
with MinNorm2) and an oracle restatement of the reference's HMC loop
(core/update.py:51-78) consume the SAME momenta, pseudofermion noise and
Metropolis uniforms; per-trajectory dH, accept/reject decisions and the
resulting chain must agree (FP64 solves at tol 1e-12 on both sides)."""

import numpy as np
import pytest

from oracle import wilson as W

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("CUDA device required", allow_module_level=True)

from jaxqft_b200.integrators import MinNorm2  # noqa: E402
from jaxqft_b200.su3_wilson_nf2 import SU3WilsonNf2  # noqa: E402
from jaxqft_b200.update import HMC  # noqa: E402


def oracle_chain(U, Ps, etas, Rs, mass, bc, beta, tol, nmd, tau, eo):
    out = []
    for P, eta, R in zip(Ps, etas, Rs):
        if eo:
            phi = W.project(W.schur_even(U, W.project(eta, 0), mass, bc, normalized=True, dag=True), 0)
        else:
            phi = W.apply_Ddag(U, eta, mass, bc)
        H0 = W.hamiltonian(U, P, phi, mass, bc, beta, tol, eo)[0]
        P1, U1 = W.minnorm2(P, U, lambda u: W.total_force(u, phi, mass, bc, beta, tol, eo), nmd, tau)
        H1 = W.hamiltonian(U1, P1, phi, mass, bc, beta, tol, eo)[0]
        dH = H1 - H0
        acc = R < (1.0 if dH < 0 else np.exp(-dH))
        if acc:
            U = U1
        out.append((dH, bool(acc), float(W.average_plaquette(U)[0])))
    return out, U


@pytest.mark.parametrize("kind", ["unpreconditioned", "eo_preconditioned"])
def test_hmc_chain_matches_oracle(kind):
    shape, beta, mass, bc, tol, nmd, tau, ntraj = (4, 4, 4, 4), 5.6, W.kappa_to_mass(0.13), (1, 1, 1, -1), 1e-12, 4, 0.5, 3
    rng = np.random.default_rng(123)
    U0 = W.hot_links(rng, shape, 1, 0.1)
    Ps = [W.algebra_field(rng, shape, 1) for _ in range(ntraj)]
    etas = [W.gaussian_spinor(rng, shape, 1) for _ in range(ntraj)]
    Rs = [float(v) for v in rng.random(ntraj)]
    # bias one uniform close to 1 so a rejection path is also exercised when dH > 0
    eo = kind == "eo_preconditioned"
    ref, Uref = oracle_chain(U0, Ps, etas, Rs, mass, bc, beta, tol, nmd, tau, eo)

    th = SU3WilsonNf2(lattice_shape=shape, beta=beta, mass=mass, fermion_bc=bc, cg_tol=tol, cg_maxiter=5000,
                      fermion_monomial_kind=kind, pseudofermion_force_mode="analytic")
    it_P, it_eta, it_R = iter(Ps), iter(etas), iter(Rs)
    th.refreshP = lambda: torch.from_numpy(next(it_P)).cuda()
    th.random_fermion = lambda: torch.from_numpy(next(it_eta)).cuda()
    hmc = HMC(th, MinNorm2(th.force, th.evolve_q, nmd, tau), verbose=False, uniform=lambda shp: [next(it_R)])
    U = torch.from_numpy(U0).cuda()
    for k in range(ntraj):
        U = hmc.evolve(U, 1)
        dH, acc = hmc.history[-1]["dH"][0], hmc.history[-1]["accepted"][0]
        rdH, racc, rplaq = ref[k]
        assert abs(dH - rdH) < 1e-8 * max(1.0, abs(rdH)), (k, dH, rdH)
        assert acc == racc, k
        assert abs(float(th.average_plaquette(U)[0]) - rplaq) < 1e-12
    assert np.linalg.norm(U.cpu().numpy() - Uref) / np.linalg.norm(Uref) < 1e-10


@pytest.fixture(scope="module")
def md_setup():
    shape, beta, mass, bc = (4, 4, 4, 4), 5.6, W.kappa_to_mass(0.13), (1, 1, 1, -1)
    rng = np.random.default_rng(5)
    U = torch.from_numpy(W.hot_links(rng, shape, 1, 0.1)).cuda()
    P = torch.from_numpy(W.algebra_field(rng, shape, 1)).cuda()
    th = SU3WilsonNf2(lattice_shape=shape, beta=beta, mass=mass, fermion_bc=bc, cg_tol=1e-13, cg_maxiter=5000,
                      pseudofermion_force_mode="analytic")
    th.fermion_monomial.refresh(U)
    return th, U, P


def _dH(th, U, P, nmd, tau):
    H0 = th.kinetic(P) + th.action(U)
    P1, U1 = MinNorm2(th.force, th.evolve_q, nmd, tau).integrate(P, U)
    return float((th.kinetic(P1) + th.action(U1) - H0)[0]), P1, U1


def test_reversibility(md_setup):
    """Integrate forward, flip the momenta, integrate again: back to the start
    (su3_wilson_nf2.py:2795-2882)."""
    th, U, P = md_setup
    _, P1, U1 = _dH(th, U, P, 5, 0.5)
    P2, U2 = MinNorm2(th.force, th.evolve_q, 5, 0.5).integrate(-P1, U1)
    assert float(torch.linalg.vector_norm(U2 - U) / torch.linalg.vector_norm(U)) < 1e-10
    assert float(torch.linalg.vector_norm(P2 + P) / torch.linalg.vector_norm(P)) < 1e-9


def test_energy_violation_scales_as_eps_squared(md_setup):
    """MinNorm2 is second order: |dH| falls ~4x when the step halves
    (su3_wilson_nf2.py:2885-2961)."""
    th, U, P = md_setup
    d = [abs(_dH(th, U, P, nmd, 0.5)[0]) for nmd in (4, 8, 16)]
    slopes = [np.log2(d[i] / d[i + 1]) for i in range(2)]
    assert all(1.6 < s < 2.4 for s in slopes), (d, slopes)


def test_identically_seeded_chains_are_bitwise_reproducible():
    """Two HMC chains with the same seeds give bit-identical dH, decisions and
    links (the reference's mcmc_smoke.py:148-200 allows 1e-7; the reductions
    here have a fixed order and no floating-point atomics, so repeats agree
    exactly)."""
    shape, mass, bc = (4, 4, 4, 4), W.kappa_to_mass(0.13), (1, 1, 1, -1)
    U0 = W.hot_links(np.random.default_rng(9), shape, 1, 0.1)

    def chain():
        th = SU3WilsonNf2(lattice_shape=shape, beta=5.6, mass=mass, fermion_bc=bc, cg_tol=1e-10, cg_maxiter=5000,
                          fermion_monomial_kind="eo_preconditioned", pseudofermion_force_mode="analytic",
                          solver_precision="half", seed=11)
        hmc = HMC(th, MinNorm2(th.force, th.evolve_q, 4, 0.5), verbose=False, seed=12)
        U = hmc.evolve(torch.from_numpy(U0).cuda(), 3)
        return [(h["dH"][0], h["accepted"][0]) for h in hmc.history], U.cpu().numpy()

    h1, U1 = chain()
    h2, U2 = chain()
    assert len(h1) == 3 and h1 == h2
    assert np.array_equal(U1, U2)
