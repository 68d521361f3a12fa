"""The C restatement (oracle/c/wilson_cpu.c) against the numpy oracle.

The C code is the CPU baseline of the bench and the checker of the full-size
GPU operator tests (24^3x48, where the numpy oracle is too slow), so it is
pinned here on small lattices against oracle/wilson.py, which the golden
vectors of the reference pin in turn: the compact hops, D and D^dag built from
them, the normalized even Schur normal operator M^dag M, and the CG iteration
count and solution of solve_eop_even_normal.
"""

import numpy as np
import pytest

from oracle import cpu as C
from oracle import wilson as W
from tests.conftest import rel

CASES = [
    ((4, 4, 4, 4), (1, 1, 1, -1), 0.12),
    ((2, 4, 6, 4), (1, 1, complex(np.cos(np.pi / 3), np.sin(np.pi / 3)), -1), 0.135),
]


@pytest.fixture(scope="module", params=range(len(CASES)))
def case(request):
    C.build()
    shape, bc, kappa = CASES[request.param]
    rng = np.random.default_rng(31 + request.param)
    U = W.hot_links(rng, shape, 1, 0.3)
    mass = W.kappa_to_mass(kappa)
    bc64 = tuple(complex(np.complex64(complex(b))) for b in bc)  # the reference builds phases in complex64
    return shape, bc64, mass, U, C.CpuWilson(U[0], shape, bc, mass), rng


def test_c_oracle_D_and_Ddag(case):
    shape, bc, mass, U, cw, rng = case
    psi = W.gaussian_spinor(rng, shape, 1)
    assert rel(cw.apply_D(psi[0]), W.apply_D(U, psi, mass, bc)[0]) < 1e-14
    assert rel(cw.apply_D(psi[0], dag=True), W.apply_Ddag(U, psi, mass, bc)[0]) < 1e-14


def test_c_oracle_schur_normal(case):
    shape, bc, mass, U, cw, rng = case
    xe = W.project(W.gaussian_spinor(rng, shape, 1), 0)
    ref = W.schur_even(U, W.schur_even(U, xe, mass, bc, normalized=True), mass, bc, normalized=True, dag=True)
    out = cw.normal(W.pack(xe, 0)[0])
    assert rel(out, W.pack(ref, 0)[0]) < 1e-14


def test_c_oracle_cg_matches_numpy_cg(case):
    shape, bc, mass, U, cw, rng = case
    b = W.project(W.gaussian_spinor(rng, shape, 1), 0)
    x_ref, its = W.solve_eop_even_normal(U, b, mass, bc, 1e-10, 1000)
    x, k, res = cw.cg(W.pack(b, 0)[0], 1e-10, 1000)
    assert res <= 1e-10
    assert k == its[0]
    assert rel(x, W.pack(x_ref, 0)[0]) < 1e-9
