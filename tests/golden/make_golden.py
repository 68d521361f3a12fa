"""Generate golden input/output vectors by running the reference's own code.

Run where the jaxQFT sources are available (pass their root with ``--ref``).
The reference modules are
imported unchanged under the numpy JAX shim (``_shim/jax``, see
``reference_loader.py``) with ``dtype=complex128``, so every output below is
what the reference's algorithm computes in FP64 on the stored inputs.

Inputs are drawn here with numpy PCG64 (seeded), not with the reference's
``jax.random`` streams: links are ``expm(TA(a*(G1 + i G2)))`` per link, which is
what ``SU3YangMills.hot_start(scale=a)`` computes (jaxqft/models/su3_ym.py:238-
247, 366-367); spinors are complex Gaussians with E|z|^2 = 1 as in
``random_fermion`` (jaxqft/models/su3_wilson_nf2.py:1169-1175).

Output: ``golden_<case>.npz`` beside this script.  Usage:
    python tests/golden/make_golden.py --ref /path/to/jaxQFT
"""

from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

CASES = {
    # 4^4, kappa=0.12 (mass = 1/(2 kappa) - 4), antiperiodic t, links hot(0.3)
    "a": dict(shape=(4, 4, 4, 4), batch=1, kappa=0.12, bc=(1, 1, 1, -1), scale=0.3, seed=0),
    # anisotropic 2x4x6x4, batch 2, kappa=0.135, phase i in z, antiperiodic t
    "b": dict(
        shape=(2, 4, 6, 4),
        batch=2,
        kappa=0.135,
        bc=(1, 1, 1j, -1),
        scale=0.2,
        seed=1,
    ),
}


def ta(x):
    y = 0.5 * (x - np.conj(np.swapaxes(x, -1, -2)))
    tr = np.trace(y, axis1=-2, axis2=-1)[..., None, None] / 3.0
    return y - tr * np.eye(3)


def gen_inputs(rng, shape, batch, scale):
    import scipy.linalg as sl

    lshape = (batch, 4, *shape, 3, 3)
    a = scale * (rng.standard_normal(lshape) + 1j * rng.standard_normal(lshape))
    U = sl.expm(ta(a))
    fshape = (batch, *shape, 4, 3)

    def spinor():
        return (rng.standard_normal(fshape) + 1j * rng.standard_normal(fshape)) / np.sqrt(2.0)

    P = ta(rng.standard_normal(lshape) + 1j * rng.standard_normal(lshape))
    return dict(U=U, psi=spinor(), chi=spinor(), X=spinor(), Y=spinor(), eta=spinor(), P=P)


def run_case(R, name, cfg):
    rng = np.random.default_rng(cfg["seed"])
    mass = 1.0 / (2.0 * cfg["kappa"]) - 4.0
    common = dict(
        lattice_shape=cfg["shape"],
        beta=5.6,
        batch_size=cfg["batch"],
        mass=mass,
        dtype=np.complex128,
        fermion_bc=tuple(complex(v) for v in cfg["bc"]),
        cg_tol=1e-12,
        cg_maxiter=5000,
        pseudofermion_force_mode="analytic",
    )
    th = R.nf2.SU3WilsonNf2(eo_use_half_spinor=False, **common)
    th_hs = R.nf2.SU3WilsonNf2(eo_use_half_spinor=True, **common)
    inp = gen_inputs(rng, cfg["shape"], cfg["batch"], cfg["scale"])
    U, psi, chi, X, Y, eta, P = (inp[k] for k in ("U", "psi", "chi", "X", "Y", "eta", "P"))
    cgmod = sys.modules["jax.scipy.sparse.linalg"]
    out = dict(inp)
    out["mass"] = np.float64(mass)
    out["bc"] = np.asarray(cfg["bc"], dtype=np.complex128)
    out["shape"] = np.asarray(cfg["shape"], dtype=np.int64)
    out["gamma"] = np.asarray(th.gamma)
    out["gamma5"] = np.asarray(R.gamma.gamma5(th.gamma))
    # index maps (jaxqft/models/su3_wilson_nf2.py:831-882)
    out["even_idx"] = np.asarray(th._cb_even_idx)
    out["odd_idx"] = np.asarray(th._cb_odd_idx)
    for k in ("plus_oe", "minus_oe", "bwd_oe", "plus_eo", "minus_eo", "bwd_eo", "target_oe", "target_eo"):
        out[k] = np.asarray(getattr(th, "_cb_" + k))
    out["mask_even"] = np.asarray(th._mask_even).reshape(cfg["shape"])
    # operators (wilson.py:171-336; su3_wilson_nf2.py:1036-1155)
    out["D_psi"] = th.apply_D(U, psi)
    out["D_psi_refkernel"] = th.apply_D_with_kernel(U, psi, kernel="reference")
    out["Ddag_psi"] = th.apply_Ddag(U, psi)
    out["N_psi"] = th.apply_normal(U, psi)
    out["offdiag_psi"] = th.apply_offdiag(U, psi)
    out["offdiag_dag_psi"] = th.apply_offdiag_dagger(U, psi)
    psi_e = th._project_even(psi)
    psi_o = th._project_odd(psi)
    out["K_oe_psi"] = th.apply_K_oe(U, psi_e)
    out["K_eo_psi"] = th.apply_K_eo(U, psi_o)
    out["Kdag_oe_psi"] = th.apply_Kdag_oe(U, psi_e)
    out["Kdag_eo_psi"] = th.apply_Kdag_eo(U, psi_o)
    out["schur_e_psi"] = th.apply_eo_schur_even(U, psi_e, normalized=False)
    out["schur_e_norm_psi"] = th.apply_eo_schur_even(U, psi_e, normalized=True)
    out["schur_e_dag_norm_psi"] = th.apply_eo_schur_even_dagger(U, psi_e, normalized=True)
    out["schur_o_norm_psi"] = th.apply_eo_schur_odd(U, psi_o, normalized=True)
    out["schur_e_compact_psi"] = th.apply_eo_schur_even_compact(U, psi_e, daggered=False, normalized=True)
    out["schur_e_compact_dag_psi"] = th.apply_eo_schur_even_compact(U, psi_e, daggered=True, normalized=True)
    out["schur_e_compact_hs_psi"] = th_hs.apply_eo_schur_even_compact(U, psi_e, daggered=False, normalized=True)
    # solves (su3_wilson_nf2.py:1370-1432) at tol 1e-12
    phi = th.apply_Ddag(U, eta)
    out["phi"] = phi
    out["solve_normal_x"] = th.solve_normal(U, phi)
    out["solve_normal_iters"] = np.int64(cgmod.cg.last_num_iters)
    phi_e = th._project_even(th.apply_eo_schur_even_dagger(U, th._project_even(eta), normalized=True))
    out["phi_e"] = phi_e
    out["solve_eop_x"] = th.solve_eop_even_normal(U, phi_e)
    out["solve_eop_iters"] = np.int64(cgmod.cg.last_num_iters)
    # pseudofermion actions (su3_wilson_nf2.py:1183-1208)
    out["pf_action"] = th.pseudofermion_action(U, phi)
    out["eop_pf_action"] = th.eop_pseudofermion_action(U, phi_e)
    # forces (su3_wilson_nf2.py:1556-1597) on arbitrary X, Y
    out["force_XY"] = th.pseudofermion_force_from_solution(U, X, Y)
    Xe = th._project_even(X)
    Ye = th._project_even(Y)
    out["eop_force_XY"] = th.eop_pseudofermion_force_from_solution(U, Xe, Ye)
    # monomial analytic forces with the refresh inputs fixed (phi given)
    mono = th.fermion_monomial
    out["mono_force_analytic"] = mono.force_analytic(U, phi)
    th_eo = R.nf2.SU3WilsonNf2(
        eo_use_half_spinor=False, fermion_monomial_kind="eo_preconditioned", **common
    )
    out["eop_mono_force_analytic"] = th_eo.fermion_monomial.force_analytic(U, phi_e)
    # gauge pieces (su3_ym.py)
    out["gauge_action"] = th.action_reference(U)
    out["gauge_force"] = R.su3_ym.SU3YangMills.force(th, U)
    out["avg_plaquette"] = th.average_plaquette(U)
    out["kinetic_P"] = th.kinetic(P)
    out["evolve_q"] = th.evolve_q(0.1, P, U)
    out["ref_flops_site_D"] = np.int64(th.dirac.flops_per_site_matvec(nc=3))
    out = {k: np.asarray(v) for k, v in out.items()}
    path = os.path.join(HERE, f"golden_{name}.npz")
    np.savez(path, **out)
    print(f"wrote {path}: {len(out)} arrays, {os.path.getsize(path)/1e6:.2f} MB, "
          f"cg iters normal={int(out['solve_normal_iters'])} eop={int(out['solve_eop_iters'])}")


def run_meas(R):
    """Point-source propagator and pion correlator through the reference's own
    measurement code (jaxqft/core/measurements.py:277-390, iterative backend,
    solver kind "cg": solve_normal(U, apply_Ddag(U, delta)) per column) on a
    4^4 lattice with an odd-parity source."""
    import importlib

    meas = importlib.import_module("jaxqft.core.measurements")
    rng = np.random.default_rng(5)
    shape, kappa, source = (4, 4, 4, 4), 0.12, (1, 0, 2, 2)
    mass = 1.0 / (2.0 * kappa) - 4.0
    th = R.nf2.SU3WilsonNf2(lattice_shape=shape, beta=5.6, batch_size=1, mass=mass, dtype=np.complex128,
                            fermion_bc=(1, 1, 1, -1), cg_tol=1e-12, cg_maxiter=5000, eo_use_half_spinor=False)
    U = gen_inputs(rng, shape, 1, 0.3)["U"]
    prop, _ = meas._full_point_source_propagator(U, th, meas.MeasurementContext(), source, backend="iterative")
    corr = meas._pion_two_point_from_propagator(np.asarray(prop), source[3])
    out = dict(U=U, mass=np.float64(mass), shape=np.asarray(shape), source=np.asarray(source),
               prop=np.asarray(prop), pion=np.asarray(corr))
    path = os.path.join(HERE, "golden_meas.npz")
    np.savez(path, **out)
    print(f"wrote {path}: prop {out['prop'].shape}, pion {out['pion']}")


def run_chrono(R):
    """Chronological initial guesses through the reference's own predictors
    (jaxqft/models/su3_wilson_nf2.py:85-194) on synthetic histories: y_i = A x_i
    for a fixed well-conditioned A, target = A (a smooth extrapolation of the
    x_i) + small noise, so that the MRE guess is accepted; a second target far
    from the image span exercises the fallback to the last solution."""
    rng = np.random.default_rng(9)
    shape = (1, 2, 2, 2, 2, 4, 3)
    n = int(np.prod(shape))
    A = np.eye(n) + 0.3 * (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) / np.sqrt(n)

    def field():
        return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) / np.sqrt(2.0)

    base, drift = field(), field()
    xs = [base + 0.1 * k * drift + 0.01 * field() for k in range(4)]
    ys = [(A @ x.reshape(-1)).reshape(shape) for x in xs]
    x_next = base + 0.4 * drift
    target = (A @ x_next.reshape(-1)).reshape(shape) + 1e-3 * field()
    far = 10.0 * field()
    out = dict(xs=np.stack(xs), ys=np.stack(ys), target=target, far=far)
    out["mre"] = np.asarray(R.nf2._chrono_predict_mre(xs, ys, target, 4))
    out["mre_far"] = np.asarray(R.nf2._chrono_predict_mre(xs, ys, far, 4))
    out["poly"] = np.asarray(R.nf2._chrono_predict_from_history(xs, "poly", 4))
    out["poly3"] = np.asarray(R.nf2._chrono_predict_from_history(xs, "poly", 3))
    out["last"] = np.asarray(R.nf2._chrono_predict_from_history(xs, "last", 4))
    path = os.path.join(HERE, "golden_chrono.npz")
    np.savez(path, **out)
    print(f"wrote {path}: mre differs from last by {np.linalg.norm(out['mre'] - out['last']):.3e}, "
          f"far fallback diff {np.linalg.norm(out['mre_far'] - out['last']):.3e}")


def run_lime(ref_root):
    """SciDAC LIME files written by jaxqft_b200.lime (gauge in D and F precision,
    one Dirac fermion) and decoded by the reference's own reader
    (jaxqft/io/lime.py decode_scidac_gauge / decode_scidac_pseudofermion)."""
    import importlib.util

    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from jaxqft_b200 import lime as ours

    spec = importlib.util.spec_from_file_location("ref_lime", os.path.join(ref_root, "jaxqft", "io", "lime.py"))
    ref = importlib.util.module_from_spec(spec)
    sys.modules["ref_lime"] = ref
    spec.loader.exec_module(ref)
    rng = np.random.default_rng(13)
    shape = (2, 4, 4, 6)
    U = gen_inputs(rng, shape, 1, 0.5)["U"][0]
    psi = (rng.standard_normal((*shape, 4, 3)) + 1j * rng.standard_normal((*shape, 4, 3))) / np.sqrt(2.0)
    out = {}
    for p in ("D", "F"):
        fn = os.path.join(HERE, f"gauge_{p}.lime")
        ours.save_gauge(fn, U, precision=p)
        out[f"U_{p}"] = ref.decode_scidac_gauge(fn)
    fn = os.path.join(HERE, "fermion_D.lime")
    ours.save_fermion(fn, psi)
    out["psi"], _ = ref.decode_scidac_pseudofermion(fn)
    out["U"], out["psi_in"] = U, psi
    np.savez(os.path.join(HERE, "golden_lime.npz"), **out)
    print("wrote LIME golden files", {k: v.shape for k, v in out.items()})


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="root of the jaxQFT source tree")
    args = ap.parse_args()
    from reference_loader import load_reference

    R = load_reference(args.ref)
    for name, cfg in CASES.items():
        run_case(R, name, cfg)
    run_meas(R)
    run_chrono(R)
    run_lime(args.ref)


if __name__ == "__main__":
    main()
