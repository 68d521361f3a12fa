"""Statistical agreement of mixed-precision and FP64 force solves in Nf=2 HMC.

    python -m jaxqft_b200.hmc_compare --shape 16,16,16,32 --therm 60 --ntraj 100

The HMC configuration (beta 5.6, kappa 0.150, MinNorm2 nmd 10, tau 1, start
exp(i*0.1*H), antiperiodic time) is first thermalised without accept/reject
(as the reference script's --warmup-no-ar), then three chains start from that
configuration:

  A  force solves with the mixed solver (FP32 or FP16 iterated operator, FP64
     reliable updates, FP64 true residual <= --cg-tol), seed s1;
  B  force solves in plain FP64 CG, seed s1 -- the same momenta, noise and
     uniforms as A, so it tracks A trajectory by trajectory;
  C  plain FP64 force solves, seed s2 -- statistically independent of A.

Every chain uses FP64 Hamiltonian solves (--action-tol) and an FP64 Metropolis
step.  Reported: per chain the acceptance, <dH>, <exp(-dH)> (1 for a correct
HMC) and <plaquette> with Gamma-method errors (jaxqft_b200.stats, the
estimator of jaxqft/testing/mcmc_smoke.py), the sigma distance of A from C for
each of them (agreement: sigma < 4, mcmc_smoke.py:135-145), and for A against
B the largest per-trajectory |dH_A - dH_B|, the number of differing accept
decisions and the largest plaquette difference.  One JSON line.
"""

from __future__ import annotations

import argparse
import json
import time

import numpy as np
import torch

from .integrators import MinNorm2
from .stats import compare_means, gamma_error
from .su3_wilson_nf2 import SU3WilsonNf2
from .update import HMC


def _theory(args, precision, seed):
    shape = tuple(int(v) for v in args.shape.split(","))
    return SU3WilsonNf2(lattice_shape=shape, beta=args.beta, mass=1.0 / (2.0 * args.kappa) - 4.0,
                        fermion_bc=(1, 1, 1, -1), cg_tol=args.cg_tol, cg_maxiter=args.cg_maxiter,
                        fermion_monomial_kind=args.monomial, pseudofermion_force_mode="analytic",
                        solver_precision=precision, action_cg_tol=args.action_tol, seed=seed)


def chain(args, U0, precision, seed, ntraj):
    th = _theory(args, precision, seed)
    hmc = HMC(th, MinNorm2(th.force, th.evolve_q, args.nmd, args.tau), verbose=False, seed=seed + 1)
    U = U0.clone()
    out = {"dH": [], "acc": [], "plaq": []}
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(ntraj):
        U = hmc.evolve(U, 1)
        h = hmc.history[-1]
        out["dH"].append(float(h["dH"][0]))
        out["acc"].append(float(bool(h["accepted"][0])))
        out["plaq"].append(float(th.average_plaquette(U)[0]))
    torch.cuda.synchronize()
    out["seconds_per_traj"] = (time.perf_counter() - t0) / max(1, ntraj)
    return out


def summary(c):
    dH = np.asarray(c["dH"])
    return {"acceptance": gamma_error(c["acc"]), "dH": gamma_error(dH), "exp_minus_dH": gamma_error(np.exp(-dH)),
            "plaquette": gamma_error(c["plaq"]), "seconds_per_traj": c["seconds_per_traj"]}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--shape", default="16,16,16,32")
    ap.add_argument("--beta", type=float, default=5.6)
    ap.add_argument("--kappa", type=float, default=0.150)
    ap.add_argument("--start-scale", type=float, default=0.1)
    ap.add_argument("--nmd", type=int, default=10)
    ap.add_argument("--tau", type=float, default=1.0)
    ap.add_argument("--therm", type=int, default=60, help="trajectories without accept/reject before the chains")
    ap.add_argument("--ntraj", type=int, default=100, help="trajectories of chains A and C")
    ap.add_argument("--ntraj-twin", type=int, default=40, help="trajectories of chain B (A's twin)")
    ap.add_argument("--monomial", default="unpreconditioned", choices=["unpreconditioned", "eo_preconditioned"])
    ap.add_argument("--precision", default="single", choices=["single", "half"], help="chain A's iterated operator")
    ap.add_argument("--cg-tol", type=float, default=1e-8)
    ap.add_argument("--action-tol", type=float, default=1e-10)
    ap.add_argument("--cg-maxiter", type=int, default=20000)
    ap.add_argument("--seeds", default="1,2")
    args = ap.parse_args(argv)
    s1, s2 = (int(v) for v in args.seeds.split(","))

    th = _theory(args, args.precision, 0)
    U = th.hot_start(scale=args.start_scale)
    integ = MinNorm2(th.force, th.evolve_q, args.nmd, args.tau)
    hmc = HMC(th, integ, verbose=False, seed=7)
    t0 = time.perf_counter()
    for _ in range(args.therm):  # refresh, integrate, always accept
        hmc._prepare_trajectory(U)
        _, U = integ.integrate(th.refreshP(), U)
    torch.cuda.synchronize()
    therm = {"trajectories": args.therm, "seconds": time.perf_counter() - t0,
             "plaquette": float(th.average_plaquette(U)[0])}
    del th, hmc, integ

    A = chain(args, U, args.precision, s1, args.ntraj)
    B = chain(args, U, "double", s1, args.ntraj_twin)
    C = chain(args, U, "double", s2, args.ntraj)
    n = args.ntraj_twin
    twin = {"trajectories": n,
            "max_abs_dH_diff": float(np.max(np.abs(np.subtract(A["dH"][:n], B["dH"][:n])))) if n else 0.0,
            "accept_decisions_differing": int(np.sum(np.asarray(A["acc"][:n]) != np.asarray(B["acc"][:n]))),
            "max_abs_plaquette_diff": float(np.max(np.abs(np.subtract(A["plaq"][:n], B["plaq"][:n])))) if n else 0.0}
    agree = {k: compare_means(a, c) for k, a, c in (
        ("acceptance", A["acc"], C["acc"]), ("dH", A["dH"], C["dH"]),
        ("exp_minus_dH", np.exp(-np.asarray(A["dH"])), np.exp(-np.asarray(C["dH"]))),
        ("plaquette", A["plaq"], C["plaq"]))}
    creutz = {name: (gamma_error(np.exp(-np.asarray(c["dH"])))["mean"] - 1.0)
              / max(gamma_error(np.exp(-np.asarray(c["dH"])))["sigma_mean"], 1e-300) for name, c in
              (("A", A), ("C", C))}
    line = {"hmc_compare": True, "shape": args.shape, "beta": args.beta, "kappa": args.kappa, "nmd": args.nmd,
            "tau": args.tau, "monomial": args.monomial, "precision_A": args.precision, "cg_tol": args.cg_tol,
            "action_tol": args.action_tol, "seeds": [s1, s2], "thermalisation": therm,
            "A": summary(A), "B": summary(B), "C": summary(C), "A_vs_B_same_seed": twin, "A_vs_C_sigma": agree,
            "exp_minus_dH_minus_1_in_sigma": creutz,
            "all_agree": bool(all(v["agree"] for v in agree.values())),
            "series": {"A": A, "C": C}}
    print(json.dumps(line), flush=True)
    return line


if __name__ == "__main__":
    main()
