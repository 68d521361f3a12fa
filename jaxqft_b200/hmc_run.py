"""Nf=2 Wilson-fermion HMC driver (the workload of the reference's
scripts/su3_wilson_nf2/hmc_su3_wilson_nf2.py) on the B200 path.

    python -m jaxqft_b200.hmc_run --shape 16,16,16,32 --beta 5.6 --kappa 0.150 \\
        --start-scale 0.1 --nmd 10 --tau 1.0 --ntraj 20 --precision single

Prints one JSON record per trajectory (dH, accept, plaquette, seconds, CG
iterations) and a summary line: acceptance, <dH>, <exp(-dH)> with its error,
plaquette history.  dH and the Metropolis step are FP64; the force solves use
the chosen inner precision with FP64 reliable updates.
"""

from __future__ import annotations

import argparse
import json
import math
import time

import numpy as np
import torch

from .integrators import ForceGradient, Leapfrog, MinNorm2
from .su3_wilson_nf2 import SU3WilsonNf2
from .update import HMC


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--shape", default="16,16,16,32")
    ap.add_argument("--beta", type=float, default=5.6)
    ap.add_argument("--kappa", type=float, default=0.150)
    ap.add_argument("--start-scale", type=float, default=0.1)
    ap.add_argument("--nmd", type=int, default=10)
    ap.add_argument("--tau", type=float, default=1.0)
    ap.add_argument("--ntraj", type=int, default=20)
    ap.add_argument("--load", default=None, help="start from a SciDAC LIME gauge configuration")
    ap.add_argument("--save", default=None, help="write the final configuration as SciDAC LIME")
    ap.add_argument("--warmup-no-ar", type=int, default=0,
                    help="initial trajectories without Metropolis accept/reject (thermalisation), as the "
                         "reference script's --warmup-no-ar")
    ap.add_argument("--integrator", default="minnorm2", choices=["minnorm2", "leapfrog", "forcegrad"])
    ap.add_argument("--monomial", default="unpreconditioned", choices=["unpreconditioned", "eo_preconditioned"])
    ap.add_argument("--precision", default="single", choices=["double", "single", "half"])
    ap.add_argument("--cg-tol", type=float, default=1e-8)
    ap.add_argument("--action-tol", type=float, default=1e-10)
    ap.add_argument("--cg-maxiter", type=int, default=20000)
    ap.add_argument("--seed", type=int, default=0)
    args = ap.parse_args(argv)
    shape = tuple(int(v) for v in args.shape.split(","))
    th = SU3WilsonNf2(lattice_shape=shape, beta=args.beta, mass=1.0 / (2.0 * args.kappa) - 4.0,
                      fermion_bc=(1, 1, 1, -1), cg_tol=args.cg_tol, cg_maxiter=args.cg_maxiter,
                      fermion_monomial_kind=args.monomial, pseudofermion_force_mode="analytic",
                      solver_precision=args.precision, action_cg_tol=args.action_tol, seed=args.seed)
    if args.load:
        from . import lime

        U = lime.load_gauge(args.load, device=th.device)
        if tuple(U.shape[2:6]) != shape:
            raise ValueError(f"{args.load}: lattice {tuple(U.shape[2:6])} differs from --shape {shape}")
    else:
        U = th.hot_start(scale=args.start_scale)
    cls = {"minnorm2": MinNorm2, "leapfrog": Leapfrog, "forcegrad": ForceGradient}[args.integrator]
    integ = cls(th.force, th.evolve_q, args.nmd, args.tau)
    hmc = HMC(th, integ, verbose=False, seed=args.seed + 1)
    # count solver iterations through the theory's solve hook
    iters = []
    orig = th._solve

    def counting_solve(*a, **k):
        out = orig(*a, **k)
        iters.extend(s["iters"] for s in th.last_solver_stats)
        return out

    th._solve = counting_solve
    plaq0 = float(th.average_plaquette(U)[0])
    for k in range(args.warmup_no_ar):
        # refresh, integrate, always accept (reference hmc_su3_wilson_nf2.py:199-213)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        hmc._prepare_trajectory(U)
        _, U = integ.integrate(th.refreshP(), U)
        torch.cuda.synchronize()
        print(json.dumps({"warmup_no_ar": k, "plaquette": float(th.average_plaquette(U)[0]),
                          "seconds": time.perf_counter() - t0}), flush=True)
    plaq_meas0 = float(th.average_plaquette(U)[0])
    records = []
    for k in range(args.ntraj):
        iters.clear()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        U = hmc.evolve(U, 1)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        h = hmc.history[-1]
        rec = {"traj": k, "dH": h["dH"][0], "accepted": bool(h["accepted"][0]),
               "plaquette": float(th.average_plaquette(U)[0]), "seconds": dt, "solves": len(iters),
               "cg_iters_total": int(sum(iters)), "cg_iters_max": int(max(iters) if iters else 0)}
        records.append(rec)
        print(json.dumps(rec), flush=True)
    dH = np.array([r["dH"] for r in records])
    ed = np.exp(-dH)
    summary = {"summary": True, "shape": shape, "beta": args.beta, "kappa": args.kappa, "nmd": args.nmd,
               "tau": args.tau, "monomial": args.monomial, "precision": args.precision, "ntraj": args.ntraj,
               "acceptance": hmc.calc_acceptance(), "mean_dH": float(dH.mean()),
               "mean_exp_minus_dH": float(ed.mean()), "err_exp_minus_dH": float(ed.std(ddof=1) / math.sqrt(len(ed)))
               if len(ed) > 1 else float("nan"), "plaquette_start": plaq0,
               "warmup_no_ar": args.warmup_no_ar, "plaquette_after_warmup": plaq_meas0,
               "plaquette_last": records[-1]["plaquette"] if records else plaq0,
               "seconds_per_traj": float(np.mean([r["seconds"] for r in records])) if records else 0.0}
    print(json.dumps(summary), flush=True)
    if args.save:
        from . import lime

        lime.save_gauge(args.save, U)
    return summary


if __name__ == "__main__":
    main()
