"""HMC with the couplings of the Nf=2 HMC configuration against the oracle chain.

beta 5.6, kappa 0.150, MinNorm2 nmd 10, tau 1, start exp(i*0.1*H), 20
trajectories on 4^4 (tests/golden/make_golden_hmc_c4.py wrote the oracle
chain: FP64 CG force solves at tol 1e-8, Hamiltonian solves at 1e-12).  The
GPU chain (jaxqft_b200.update.HMC driving SU3WilsonNf2 with MinNorm2) consumes
the same momenta, noise and uniforms and runs the force solves as the
production configuration does -- FP32 iterated operator with FP64 reliable
updates, true residual 1e-8 -- and the Hamiltonian in FP64 with 1e-12 solves.
Per trajectory dH must agree to 1e-5 absolute (force solutions at tol 1e-8
differ between the two solvers by at most cond(D^dag D) * 1e-8 ~ 1e-6
relative), the accept decisions must be the same and the plaquettes agree to
1e-8.  Both monomials (unpreconditioned, even-odd preconditioned).
"""

import os
import sys

import numpy as np
import pytest

from tests.conftest import GOLDEN

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("CUDA device required", allow_module_level=True)

sys.path.insert(0, GOLDEN)
import make_golden_hmc_c4 as G  # noqa: E402

from jaxqft_b200.integrators import MinNorm2  # noqa: E402
from jaxqft_b200.su3_wilson_nf2 import SU3WilsonNf2  # noqa: E402
from jaxqft_b200.update import HMC  # noqa: E402


@pytest.fixture(scope="module")
def golden():
    with np.load(os.path.join(GOLDEN, "golden_hmc_c4.npz")) as z:
        g = {k: z[k] for k in z.files}
    U0, Ps, etas, Rs = G.inputs(int(g["seed"]))
    np.testing.assert_allclose(G.checksums(U0, Ps, etas, Rs), g["checksums"], rtol=1e-13)
    return g, (U0, Ps, etas, Rs)


@pytest.mark.parametrize("kind", ["unpreconditioned", "eo_preconditioned"])
def test_c4_chain_matches_oracle(golden, kind):
    g, (U0, Ps, etas, Rs) = golden
    name = "eo" if kind == "eo_preconditioned" else "unprec"
    th = SU3WilsonNf2(lattice_shape=G.SHAPE, beta=G.BETA, mass=1.0 / (2.0 * G.KAPPA) - 4.0, fermion_bc=G.BC,
                      cg_tol=G.FORCE_TOL, action_cg_tol=G.ACTION_TOL, cg_maxiter=20000, fermion_monomial_kind=kind,
                      pseudofermion_force_mode="analytic", solver_precision="single")
    it_P, it_eta, it_R = iter(Ps), iter(etas), iter(Rs)
    th.refreshP = lambda: torch.from_numpy(next(it_P)).cuda()
    th.random_fermion = lambda: torch.from_numpy(next(it_eta)).cuda()
    hmc = HMC(th, MinNorm2(th.force, th.evolve_q, G.NMD, G.TAU), verbose=False, uniform=lambda shp: [next(it_R)])
    U = torch.from_numpy(U0).cuda()
    errs = []
    for k in range(G.NTRAJ):
        U = hmc.evolve(U, 1)
        dH, acc = hmc.history[-1]["dH"][0], bool(hmc.history[-1]["accepted"][0])
        rdH, racc, rplaq = g[f"{name}_dH"][k], bool(g[f"{name}_acc"][k]), g[f"{name}_plaq"][k]
        plaq = float(th.average_plaquette(U)[0])
        errs.append(abs(dH - rdH))
        assert abs(dH - rdH) < 1e-5, (k, dH, rdH)
        assert acc == racc, (k, dH, rdH)
        assert abs(plaq - rplaq) < 1e-8, (k, plaq, rplaq)
    print(f"{kind}: max |dH - dH_oracle| = {max(errs):.2e}, acceptance {np.mean(g[name + '_acc']):.2f}")
