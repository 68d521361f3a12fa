"""Chronological initial guesses inside an MD trajectory on the GPU: with the
history predictors (last / poly / MRE, su3_wilson_nf2.py:85-194, 254-294) the
force solves need fewer CG iterations, and the trajectory is the same as
without guesses to well below the solver tolerance."""

import numpy as np
import pytest

from oracle import wilson as W
from tests.conftest import rel

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("CUDA device required", allow_module_level=True)

from jaxqft_b200.integrators import MinNorm2  # noqa: E402
from jaxqft_b200.su3_wilson_nf2 import SU3WilsonNf2  # noqa: E402


def _trajectory(th, U, P):
    iters = []
    orig = th._solve

    def counting(*a, **k):
        out = orig(*a, **k)
        iters.extend(s["iters"] for s in th.last_solver_stats)
        return out

    th._solve = counting
    try:
        P1, U1 = MinNorm2(th.force, th.evolve_q, 8, 0.5).integrate(P, U)
    finally:
        th._solve = orig
    return U1, sum(iters)


@pytest.mark.parametrize("kind", ["unpreconditioned", "eo_preconditioned"])
@pytest.mark.parametrize("mode", ["last", "poly", "mre"])
def test_guesses_cut_iterations_same_trajectory(kind, mode):
    shape = (4, 4, 4, 8)
    rng = np.random.default_rng(31)
    U = torch.from_numpy(W.hot_links(rng, shape, 1, 0.2)).cuda()
    P = torch.from_numpy(W.algebra_field(rng, shape, 1)).cuda()
    th = SU3WilsonNf2(lattice_shape=shape, beta=5.6, mass=-0.2, fermion_bc=(1, 1, 1, -1), cg_tol=1e-11,
                      cg_maxiter=5000, fermion_monomial_kind=kind, pseudofermion_force_mode="analytic",
                      solver_precision="single", use_solver_guess=True, solver_guess_mode=mode,
                      solver_guess_history=4, seed=3)
    th.prepare_trajectory(U)  # heatbath: eta and phi
    mono = th.fermion_monomial
    assert mono.eta is not None
    U_g, it_g = _trajectory(th, U, P)
    th.use_solver_guess = False
    mono.clear_solver_guess()
    U_0, it_0 = _trajectory(th, U, P)
    assert it_g < it_0, (mode, it_g, it_0)
    assert rel(U_g.cpu().numpy(), U_0.cpu().numpy()) < 1e-9


def test_device_predictors_match_reference():
    """The predictors on the library's kernels (wl_field_dots / wl_field_combine)
    against the reference's own outputs (golden_chrono.npz)."""
    from jaxqft_b200.lib import WilsonContext
    from jaxqft_b200.su3_wilson_nf2 import _chrono_predict, _chrono_predict_mre, _DeviceAlgebra
    from tests.conftest import load_golden

    g = load_golden("chrono")
    la = _DeviceAlgebra(WilsonContext((4, 4, 4, 4)))
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    xs, ys = [t(x) for x in g["xs"]], [t(y) for y in g["ys"]]
    assert rel(_chrono_predict(xs, "poly", 4, la=la).cpu().numpy(), g["poly"]) < 1e-14
    assert rel(_chrono_predict(xs, "poly", 3, la=la).cpu().numpy(), g["poly3"]) < 1e-14
    assert rel(_chrono_predict_mre(xs, ys, t(g["target"]), la=la).cpu().numpy(), g["mre"]) < 1e-12
    assert rel(_chrono_predict_mre(xs, ys, t(g["far"]), la=la).cpu().numpy(), g["mre_far"]) < 1e-15
    d = la.dots([(xs[0], ys[1]), (ys[2], ys[2])])
    assert abs(d[0] - np.vdot(g["xs"][0], g["ys"][1])) < 1e-12 * abs(d[0])
    assert abs(d[1] - np.vdot(g["ys"][2], g["ys"][2])) < 1e-12 * abs(d[1])


def test_device_predictors_match_reference():
    """The predictors on the library's kernels (wl_field_dots / wl_field_combine)
    against the reference's own outputs (golden_chrono.npz)."""
    from jaxqft_b200.lib import WilsonContext
    from jaxqft_b200.su3_wilson_nf2 import _chrono_predict, _chrono_predict_mre, _DeviceAlgebra
    from tests.conftest import load_golden

    g = load_golden("chrono")
    la = _DeviceAlgebra(WilsonContext((4, 4, 4, 4)))
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    xs, ys = [t(x) for x in g["xs"]], [t(y) for y in g["ys"]]
    assert rel(_chrono_predict(xs, "poly", 4, la=la).cpu().numpy(), g["poly"]) < 1e-14
    assert rel(_chrono_predict(xs, "poly", 3, la=la).cpu().numpy(), g["poly3"]) < 1e-14
    assert rel(_chrono_predict_mre(xs, ys, t(g["target"]), la=la).cpu().numpy(), g["mre"]) < 1e-12
    assert rel(_chrono_predict_mre(xs, ys, t(g["far"]), la=la).cpu().numpy(), g["mre_far"]) < 1e-15
    d = la.dots([(xs[0], ys[1]), (ys[2], ys[2])])
    assert abs(d[0] - np.vdot(g["xs"][0], g["ys"][1])) < 1e-12 * abs(d[0])
    assert abs(d[1] - np.vdot(g["ys"][2], g["ys"][2])) < 1e-12 * abs(d[1])
