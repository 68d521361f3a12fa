"""The drop-in theory API (jaxqft_b200.SU3WilsonNf2) against the reference's
golden vectors and the oracle: every apply/solve/action/force method on the
reference's own inputs, and one full MinNorm2 molecular-dynamics trajectory
(gauge + pseudofermion forces, exponential drift) against the oracle."""

import numpy as np
import pytest

from oracle import wilson as W
from tests.conftest import load_golden, rel

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("CUDA device required", allow_module_level=True)

from jaxqft_b200.integrators import MinNorm2  # noqa: E402
from jaxqft_b200.su3_wilson_nf2 import SU3WilsonNf2  # noqa: E402

TOL = 1e-13


def make(g, **kw):
    return SU3WilsonNf2(lattice_shape=tuple(int(v) for v in g["shape"]), beta=5.6, batch_size=g["U"].shape[0],
                        mass=float(g["mass"]), fermion_bc=tuple(g["bc"]), cg_tol=1e-12, cg_maxiter=5000,
                        pseudofermion_force_mode="analytic", **kw)


@pytest.fixture(scope="module", params=["a", "b"])
def case(request):
    return load_golden(request.param)


def n(t):
    return t.detach().cpu().numpy()


def test_operators(case):
    g = case
    th = make(g)
    U, psi = g["U"], g["psi"]
    pe, po = W.project(psi, 0), W.project(psi, 1)
    checks = {
        "D_psi": th.apply_D(U, psi), "Ddag_psi": th.apply_Ddag(U, psi), "N_psi": th.apply_normal(U, psi),
        "offdiag_psi": th.apply_offdiag(U, psi), "offdiag_dag_psi": th.apply_offdiag_dagger(U, psi),
        "K_oe_psi": th.apply_K_oe(U, pe), "K_eo_psi": th.apply_K_eo(U, po),
        "Kdag_oe_psi": th.apply_Kdag_oe(U, pe), "Kdag_eo_psi": th.apply_Kdag_eo(U, po),
        "schur_e_psi": th.apply_eo_schur_even(U, pe), "schur_e_norm_psi": th.apply_eo_schur_even(U, pe, True),
        "schur_e_dag_norm_psi": th.apply_eo_schur_even_dagger(U, pe, True),
        "schur_o_norm_psi": th.apply_eo_schur_odd(U, po, True),
        "schur_e_compact_psi": th.apply_eo_schur_even_compact(U, pe),
        "schur_e_compact_dag_psi": th.apply_eo_schur_even_compact(U, pe, daggered=True),
    }
    for k, v in checks.items():
        assert rel(n(v), g[k]) < TOL, k
    # EO helpers: pack/unpack round trip and masks
    pk = th._pack_even_sites(pe)
    assert rel(n(th._unpack_even_sites(pk)), pe) == 0.0


def test_solves_actions_and_forces(case):
    g = case
    th = make(g)
    U = g["U"]
    x = th.solve_normal(U, g["phi"])
    assert rel(n(x), g["solve_normal_x"]) < 1e-9
    assert all(s["status"] == 2 for s in th.last_solver_stats)
    xe = th.solve_eop_even_normal(U, g["phi_e"])
    assert rel(n(xe), g["solve_eop_x"]) < 1e-9
    assert np.allclose(n(th.pseudofermion_action(U, g["phi"])), g["pf_action"], rtol=1e-10)
    assert np.allclose(n(th.eop_pseudofermion_action(U, g["phi_e"])), g["eop_pf_action"], rtol=1e-10)
    assert rel(n(th.pseudofermion_force_from_solution(U, g["X"], g["Y"])), g["force_XY"]) < TOL
    assert rel(n(th.eop_pseudofermion_force_from_solution(U, W.project(g["X"], 0), W.project(g["Y"], 0))),
               g["eop_force_XY"]) < TOL
    mono = th.fermion_monomial
    assert rel(n(mono.force_analytic(U, torch.from_numpy(g["phi"]).cuda())), g["mono_force_analytic"]) < 1e-9
    th_eo = make(g, fermion_monomial_kind="eo_preconditioned")
    assert rel(n(th_eo.fermion_monomial.force_analytic(U, torch.from_numpy(g["phi_e"]).cuda())),
               g["eop_mono_force_analytic"]) < 1e-9


def test_gauge_pieces(case):
    g = case
    th = make(g)
    U = torch.from_numpy(g["U"]).cuda()
    assert np.allclose(n(th.gauge_action(U)), g["gauge_action"], rtol=1e-12)
    assert rel(n(th.gauge_force(U)), g["gauge_force"]) < 1e-13
    assert np.allclose(n(th.average_plaquette(U)), g["avg_plaquette"], rtol=1e-12)
    assert np.allclose(n(th.kinetic(torch.from_numpy(g["P"]).cuda())), g["kinetic_P"], rtol=1e-12)
    assert rel(n(th.evolve_q(0.1, torch.from_numpy(g["P"]).cuda(), U)), g["evolve_q"]) < 1e-13


@pytest.mark.parametrize("kind", ["unpreconditioned", "eo_preconditioned"])
@pytest.mark.parametrize("prec", ["double", "single"])
def test_md_trajectory_matches_oracle(kind, prec):
    """Same U, P and pseudofermion: one MinNorm2 trajectory (nmd=3, tau=0.3)
    through theory.force / theory.evolve_q against the oracle's integration.
    FP32 inner solves differ from FP64 only below the 1e-12 solver tolerance."""
    shape = (4, 4, 4, 4)
    rng = np.random.default_rng(77)
    U = W.hot_links(rng, shape, 1, 0.2)
    P = W.algebra_field(rng, shape, 1)
    mass, bc, beta, tol = -0.2, (1, 1, 1, -1), 5.6, 1e-12
    eo = kind == "eo_preconditioned"
    eta = W.gaussian_spinor(rng, shape, 1)
    if eo:
        phi = W.project(W.schur_even(U, W.project(eta, 0), mass, bc, normalized=True, dag=True), 0)
    else:
        phi = W.apply_Ddag(U, eta, mass, bc)
    th = SU3WilsonNf2(lattice_shape=shape, beta=beta, mass=mass, fermion_bc=bc, cg_tol=tol, cg_maxiter=5000,
                      fermion_monomial_kind=kind, pseudofermion_force_mode="analytic", solver_precision=prec)
    th.set_loaded_pseudofermion(torch.from_numpy(phi).cuda())
    Ut, Pt = torch.from_numpy(U).cuda(), torch.from_numpy(P).cuda()
    H0 = th.kinetic(Pt) + th.action(Ut)
    integ = MinNorm2(th.force, th.evolve_q, 3, 0.3)
    P1, U1 = integ.integrate(Pt, Ut)
    H1 = th.kinetic(P1) + th.action(U1)
    Pr, Ur = W.minnorm2(P, U, lambda u: W.total_force(u, phi, mass, bc, beta, tol, eo), 3, 0.3)
    H0r = W.hamiltonian(U, P, phi, mass, bc, beta, tol, eo)
    H1r = W.hamiltonian(Ur, Pr, phi, mass, bc, beta, tol, eo)
    assert rel(n(U1), Ur) < 1e-10
    assert rel(n(P1), Pr) < 1e-9
    dh, dhr = float((H1 - H0)[0]), float((H1r - H0r)[0])
    assert abs(dh - dhr) < 1e-7 * max(1.0, abs(dhr))
