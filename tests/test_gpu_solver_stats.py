"""The solver diagnostics of the drop-in theory (su3_wilson_nf2.py:1456-1554).

normal_residual_stats: the relative and absolute residuals of (D^dag D) x = phi,
recomputed here with the numpy oracle on the same fields.  solver_info_stats:
real per-RHS iteration counts -- for the normal form equal (to one iteration,
the FP64 engine checks its true residual only when the recursive one converges)
to the oracle's restatement of the CG the reference runs; for the split forms
the stage-1 (A^dag y = phi) and stage-2 (A x = y) means add up to the total.
"""

import math

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
MASS = W.kappa_to_mass(0.13)


@pytest.fixture(scope="module")
def fields():
    rng = np.random.default_rng(77)
    return W.hot_links(rng, SHAPE, 2, 0.2), W.gaussian_spinor(rng, SHAPE, 2)


def test_normal_residual_stats_match_oracle(fields):
    U, phi = fields
    th = SU3WilsonNf2(lattice_shape=SHAPE, beta=5.6, mass=MASS, fermion_bc=BC, cg_tol=1e-6, batch_size=2,
                      solver_precision="double")
    Ut, pt = torch.from_numpy(U).cuda(), torch.from_numpy(phi).cuda()
    x = th.solve_normal(Ut, pt)  # a loose solve: residuals well above rounding
    st = th.normal_residual_stats(Ut, pt, x)
    r = W.apply_normal(U, x.cpu().numpy(), MASS, BC) - phi
    rel = [np.linalg.norm(r[b]) / (np.linalg.norm(phi[b]) + 1e-30) for b in range(2)]
    absn = [np.linalg.norm(r[b]) for b in range(2)]
    ref = {"mean_rel_residual": np.mean(rel), "max_rel_residual": np.max(rel),
           "mean_abs_residual": np.mean(absn), "max_abs_residual": np.max(absn)}
    for k, v in ref.items():
        assert abs(st[k] - v) <= 1e-8 * v, (k, st[k], v)
    assert st["max_rel_residual"] <= 1e-6


def test_solver_info_stats_normal_matches_oracle_cg(fields):
    U, phi = fields
    th = SU3WilsonNf2(lattice_shape=SHAPE, beta=5.6, mass=MASS, fermion_bc=BC, cg_tol=1e-10, batch_size=2,
                      solver_precision="double", cg_maxiter=5000)
    st = th.solver_info_stats(torch.from_numpy(U).cuda(), torch.from_numpy(phi).cuda())
    _, its = W.solve_normal(U, phi, MASS, BC, 1e-10, 5000)
    assert st["iters_known_fraction"] == 1.0
    assert abs(st["mean_solver_iters"] - np.mean(its)) <= 1.0, (st, its)
    assert abs(st["max_solver_iters"] - np.max(its)) <= 1.0, (st, its)
    assert math.isnan(st["mean_solver_iters_stage1"]) and math.isnan(st["mean_solver_iters_stage2"])


@pytest.mark.parametrize("form", ["split", "eo_split"])
def test_solver_info_stats_split_stages(fields, form):
    U, phi = fields
    th = SU3WilsonNf2(lattice_shape=SHAPE, beta=5.6, mass=MASS, fermion_bc=BC, cg_tol=1e-9, batch_size=2,
                      solver_kind="bicgstab", solver_form=form, solver_precision="single", cg_maxiter=5000)
    st = th.solver_info_stats(torch.from_numpy(U).cuda(), torch.from_numpy(phi).cuda())
    assert st["iters_known_fraction"] == 1.0
    assert st["mean_solver_iters_stage1"] > 0 and st["mean_solver_iters_stage2"] > 0
    assert abs(st["mean_solver_iters_stage1"] + st["mean_solver_iters_stage2"] - st["mean_solver_iters"]) < 1e-9
