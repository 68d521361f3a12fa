"""Oracle HMC chains with the couplings of the Nf=2 HMC configuration.

beta 5.6, kappa 0.150 (bare mass 1/(2 kappa) - 4), antiperiodic time, start
links exp(i*0.1*H), MinNorm2 with nmd 10 and tau 1, 20 trajectories, force
solves at tol 1e-8 and Hamiltonian (Metropolis) solves at 1e-12, both
monomials (unpreconditioned phi = D^dag eta; even-odd phi_e = M^dag eta_e) --
on a 4^4 lattice, where the numpy oracle (oracle/wilson.py: minnorm2,
total_force, hamiltonian; the HMC loop of jaxqft/core/update.py:51-78) runs a
chain in minutes.  Inputs (start links, per-trajectory momenta, pseudofermion
noise, Metropolis uniforms) are drawn from numpy PCG64 with the seed stored in
the fixture; tests regenerate them and check the stored checksums first.

Output: ``golden_hmc_c4.npz`` beside this script (per monomial: dH, accept
decisions and plaquette after each trajectory).  Usage:
    python tests/golden/make_golden_hmc_c4.py
"""

from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import wilson as W  # noqa: E402

SHAPE = (4, 4, 4, 4)
BETA = 5.6
KAPPA = 0.150
BC = (1, 1, 1, -1)
NMD, TAU, NTRAJ = 10, 1.0, 20
FORCE_TOL, ACTION_TOL = 1e-8, 1e-12
SEED = 2024


def inputs(seed=SEED):
    """Start links, momenta, noise and uniforms of the chain (same draws on every machine)."""
    rng = np.random.default_rng(seed)
    U0 = W.hot_links(rng, SHAPE, 1, 0.1)
    Ps = [W.algebra_field(rng, SHAPE, 1) for _ in range(NTRAJ)]
    etas = [W.gaussian_spinor(rng, SHAPE, 1) for _ in range(NTRAJ)]
    Rs = [float(v) for v in rng.random(NTRAJ)]
    return U0, Ps, etas, Rs


def checksums(U0, Ps, etas, Rs):
    return np.array([np.sum(U0).real, np.sum(U0).imag, sum(np.sum(P).imag for P in Ps),
                     sum(np.sum(np.abs(e) ** 2) for e in etas), sum(Rs)])


def oracle_chain(U, Ps, etas, Rs, eo):
    mass = W.kappa_to_mass(KAPPA)
    out = []
    for P, eta, R in zip(Ps, etas, Rs):
        if eo:
            phi = W.project(W.schur_even(U, W.project(eta, 0), mass, BC, normalized=True, dag=True), 0)
        else:
            phi = W.apply_Ddag(U, eta, mass, BC)
        H0 = W.hamiltonian(U, P, phi, mass, BC, BETA, ACTION_TOL, eo)[0]
        P1, U1 = W.minnorm2(P, U, lambda u: W.total_force(u, phi, mass, BC, BETA, FORCE_TOL, eo), NMD, TAU)
        H1 = W.hamiltonian(U1, P1, phi, mass, BC, BETA, ACTION_TOL, eo)[0]
        dH = float(H1 - H0)
        acc = bool(R < (1.0 if dH < 0 else np.exp(-dH)))
        if acc:
            U = U1
        out.append((dH, acc, float(W.average_plaquette(U)[0])))
        print(f"  eo={eo} dH={dH:+.6e} acc={acc} plaq={out[-1][2]:.10f}", flush=True)
    return out


def main():
    U0, Ps, etas, Rs = inputs()
    res = {"seed": np.int64(SEED), "checksums": checksums(U0, Ps, etas, Rs),
           "params": np.array([BETA, KAPPA, NMD, TAU, FORCE_TOL, ACTION_TOL, NTRAJ])}
    for name, eo in (("unprec", False), ("eo", True)):
        t0 = time.time()
        ch = oracle_chain(U0, Ps, etas, Rs, eo)
        res[f"{name}_dH"] = np.array([c[0] for c in ch])
        res[f"{name}_acc"] = np.array([c[1] for c in ch])
        res[f"{name}_plaq"] = np.array([c[2] for c in ch])
        print(f"{name}: {time.time() - t0:.0f} s, acceptance {np.mean(res[name + '_acc']):.2f}", flush=True)
    np.savez_compressed(os.path.join(HERE, "golden_hmc_c4.npz"), **res)


if __name__ == "__main__":
    main()
