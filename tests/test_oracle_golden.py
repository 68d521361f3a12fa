"""The CPU oracle against golden vectors produced by the reference's own code
(tests/golden/make_golden.py) -- pins the oracle before it is trusted."""

import numpy as np
import pytest

from oracle import wilson as W
from tests.conftest import load_golden, rel

TOL = 1e-13


def test_gamma_basis_and_gamma5(golden):
    assert np.array_equal(W.GAMMA, golden["gamma"])
    assert np.array_equal(W.GAMMA5, golden["gamma5"])
    for mu in range(4):
        for nu in range(4):
            anti = W.GAMMA[mu] @ W.GAMMA[nu] + W.GAMMA[nu] @ W.GAMMA[mu]
            assert np.allclose(anti, 2.0 * np.eye(4) * (mu == nu))


def test_eo_maps_bit_exact(golden):
    shape = tuple(golden["shape"])
    even, odd = W.cb_indices(shape)
    assert np.array_equal(even, golden["even_idx"]) and np.array_equal(odd, golden["odd_idx"])
    maps = W.cb_neighbor_maps(shape)
    for k, v in maps.items():
        assert np.array_equal(v, golden[k]), k
        assert v.dtype == golden[k].dtype


@pytest.mark.parametrize("name,fn", [
    ("D_psi", lambda g: W.apply_D(g["U"], g["psi"], float(g["mass"]), g["bc"])),
    ("D_psi_refkernel", lambda g: W.apply_D(g["U"], g["psi"], float(g["mass"]), g["bc"])),
    ("Ddag_psi", lambda g: W.apply_Ddag(g["U"], g["psi"], float(g["mass"]), g["bc"])),
    ("N_psi", lambda g: W.apply_normal(g["U"], g["psi"], float(g["mass"]), g["bc"])),
    ("offdiag_psi", lambda g: W.apply_hop(g["U"], g["psi"], g["bc"])),
    ("offdiag_dag_psi", lambda g: W.apply_hop(g["U"], g["psi"], g["bc"], dag=True)),
    ("K_oe_psi", lambda g: W.K_block(g["U"], W.project(g["psi"], 0), g["bc"], 0)),
    ("K_eo_psi", lambda g: W.K_block(g["U"], W.project(g["psi"], 1), g["bc"], 1)),
    ("Kdag_oe_psi", lambda g: W.K_block(g["U"], W.project(g["psi"], 0), g["bc"], 0, dag=True)),
    ("Kdag_eo_psi", lambda g: W.K_block(g["U"], W.project(g["psi"], 1), g["bc"], 1, dag=True)),
    ("schur_e_psi", lambda g: W.schur_even(g["U"], W.project(g["psi"], 0), float(g["mass"]), g["bc"])),
    ("schur_e_norm_psi", lambda g: W.schur_even(g["U"], W.project(g["psi"], 0), float(g["mass"]), g["bc"], True)),
    ("schur_e_dag_norm_psi",
     lambda g: W.schur_even(g["U"], W.project(g["psi"], 0), float(g["mass"]), g["bc"], True, True)),
    ("schur_o_norm_psi", lambda g: W.schur_odd(g["U"], W.project(g["psi"], 1), float(g["mass"]), g["bc"], True)),
])
def test_operators_match_reference(golden, name, fn):
    assert rel(fn(golden), golden[name]) < TOL


def test_compact_schur_matches_reference(golden):
    g = golden
    shape = tuple(g["shape"])
    pe = W.project(g["psi"], 0)
    for dag, key in ((False, "schur_e_compact_psi"), (True, "schur_e_compact_dag_psi")):
        out = W.unpack(W.schur_even_compact(g["U"], W.pack(pe, 0), float(g["mass"]), g["bc"], shape, dag=dag),
                       shape, 0)
        assert rel(out, g[key]) < TOL
    # the reference's default half-spinor factors are built with a complex64 SVD
    # (jaxqft/fermions/wilson.py:77-105): documented ~1e-8 deviation from FP64
    out = W.unpack(W.schur_even_compact(g["U"], W.pack(pe, 0), float(g["mass"]), g["bc"], shape), shape, 0)
    assert 1e-12 < rel(out, g["schur_e_compact_hs_psi"]) < 1e-6


def test_cg_matches_reference_iterates(golden):
    g = golden
    m, bc = float(g["mass"]), g["bc"]
    x, its = W.solve_normal(g["U"], g["phi"], m, bc, 1e-12, 5000)
    assert rel(x, g["solve_normal_x"]) < 1e-12
    assert its[-1] == int(g["solve_normal_iters"])
    xe, its = W.solve_eop_even_normal(g["U"], g["phi_e"], m, bc, 1e-12, 5000)
    assert rel(xe, g["solve_eop_x"]) < 1e-12
    assert its[-1] == int(g["solve_eop_iters"])


def test_pf_action_and_forces(golden):
    g = golden
    m, bc = float(g["mass"]), g["bc"]
    assert np.allclose(W.pseudofermion_action(g["U"], g["phi"], m, bc, 1e-12, 5000), g["pf_action"], rtol=1e-12)
    assert np.allclose(W.eop_pseudofermion_action(g["U"], g["phi_e"], m, bc, 1e-12, 5000), g["eop_pf_action"],
                       rtol=1e-12)
    assert rel(W.force_from_solution(g["U"], g["X"], g["Y"], bc), g["force_XY"]) < TOL
    assert rel(W.eop_force_from_solution(g["U"], W.project(g["X"], 0), W.project(g["Y"], 0), m, bc),
               g["eop_force_XY"]) < TOL


def test_monomial_analytic_forces(golden):
    g = golden
    m, bc = float(g["mass"]), g["bc"]
    x, _ = W.solve_normal(g["U"], g["phi"], m, bc, 1e-12, 5000)
    y = W.apply_D(g["U"], x, m, bc)
    assert rel(W.force_from_solution(g["U"], x, y, bc), g["mono_force_analytic"]) < 1e-10
    xe, _ = W.solve_eop_even_normal(g["U"], g["phi_e"], m, bc, 1e-12, 5000)
    ye = W.schur_even(g["U"], xe, m, bc, normalized=True)
    assert rel(W.eop_force_from_solution(g["U"], xe, ye, m, bc), g["eop_mono_force_analytic"]) < 1e-10


def test_gauge_pieces(golden):
    g = golden
    assert np.allclose(W.gauge_action(g["U"], 5.6), g["gauge_action"], rtol=1e-13)
    assert rel(W.gauge_force(g["U"], 5.6), g["gauge_force"]) < TOL
    assert np.allclose(W.average_plaquette(g["U"]), g["avg_plaquette"], rtol=1e-13)
    assert np.allclose(W.kinetic(g["P"]), g["kinetic_P"], rtol=1e-13)
    assert rel(W.evolve_q(0.1, g["P"], g["U"]), g["evolve_q"]) < TOL


def test_free_field_stencil_known_answer():
    """Known-answer test of su3_wilson_nf2.py:2040-2082: with unit links, D is the
    free Wilson stencil with the boundary phase on the wrapping hops."""
    shape = (4, 2, 2, 6)
    rng = np.random.default_rng(5)
    psi = W.gaussian_spinor(rng, shape, 1)
    U = np.broadcast_to(np.eye(3, dtype=np.complex128), (1, 4, *shape, 3, 3)).copy()
    bc = (1, 1, 1, -1)
    mass = 0.1
    ref = (mass + 4) * psi
    for mu in range(4):
        fwd = np.roll(psi, -1, axis=1 + mu)
        bwd = np.roll(psi, +1, axis=1 + mu)
        if bc[mu] != 1:
            sl = [slice(None)] * psi.ndim
            sl[1 + mu] = shape[mu] - 1
            fwd[tuple(sl)] *= bc[mu]
            sl[1 + mu] = 0
            bwd[tuple(sl)] *= np.conj(bc[mu])
        ref = ref - 0.5 * ((fwd - W.spin_mul(W.GAMMA[mu], fwd)) + (bwd + W.spin_mul(W.GAMMA[mu], bwd)))
    assert rel(W.apply_D(U, psi, mass, bc), ref) < 1e-15


def test_gamma5_hermiticity_and_adjoint():
    shape = (4, 4, 2, 4)
    rng = np.random.default_rng(6)
    U = W.hot_links(rng, shape, 1, 0.3)
    psi, chi = W.gaussian_spinor(rng, shape, 1), W.gaussian_spinor(rng, shape, 1)
    bc = (1, 1, 1, -1)
    lhs = W.apply_Ddag(U, psi, 0.05, bc)
    rhs = W.spin_mul(W.GAMMA5, W.apply_D(U, W.spin_mul(W.GAMMA5, psi), 0.05, bc))
    assert rel(lhs, rhs) < 1e-14
    a = W.vdot(chi, W.apply_D(U, psi, 0.05, bc))
    b = W.vdot(W.apply_Ddag(U, chi, 0.05, bc), psi)
    assert abs(a - b) / abs(a) < 1e-14


def test_point_propagator_and_pion_match_reference():
    """Oracle vs the reference's own measurement code (golden_meas.npz)."""
    g = load_golden("meas")
    prop = W.point_source_propagator(g["U"], float(g["mass"]), (1, 1, 1, -1), tuple(g["source"]))
    assert rel(prop, g["prop"]) < 1e-10
    assert np.allclose(W.pion_two_point(g["prop"], int(g["source"][3])), g["pion"], rtol=1e-13, atol=0)
