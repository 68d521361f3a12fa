"""Point-source propagators and the pion two-point function on the B200 path,
mirroring ``jaxqft/core/measurements.py`` (iterative backend with the CG
solver kind, 277-372; pion contraction 375-390).

The reference solves the 12 (spin, colour) point sources one at a time through
``solve_normal(U, apply_Ddag(U, delta))``; here all 12 right-hand sides of a
configuration go through ONE batched mixed-precision solve (FP64 true residual
<= tol for every column), and the contraction runs as a device kernel
(``wl_pion_correlator``).  ``method="eo"`` solves the even-odd Schur system
and reconstructs the odd sites (su3_wilson_nf2.py:1301-1336 ``_solve_eo_one``):
the same propagator to solver tolerance, at about half the work.
"""

from __future__ import annotations

import time
from typing import Dict, Optional, Sequence, Tuple

import numpy as np
import torch

from . import lib as L


def _parity_masks(shape, device):
    x = [torch.arange(n, device=device) for n in shape]
    par = (x[0][:, None, None, None] + x[1][None, :, None, None] + x[2][None, None, :, None]
           + x[3][None, None, None, :]) % 2
    even = (par == 0).to(torch.complex128)[..., None, None]
    return even, 1.0 - even


def point_sources(shape, source: Sequence[int], device) -> torch.Tensor:
    """The 12 unit sources delta(x, source) delta(spin, s) delta(colour, c), column k = 3 s + c."""
    src = tuple(int(v) % int(n) for v, n in zip(source, shape))
    eta = torch.zeros((12, *shape, 4, 3), dtype=torch.complex128, device=device)
    for k in range(12):
        eta[(k, *src, k // 3, k % 3)] = 1.0
    return eta


def propagator_columns(ctx: L.WilsonContext, gauge: L.Gauge, mass: float, eta: torch.Tensor, *,
                       method: str = "normal", inner: str = "single", tol: float = 1e-10,
                       maxiter: int = 10000) -> Tuple[torch.Tensor, list]:
    """x_k = D^{-1} eta_k for a batch of sources eta [n, *L, 4, 3] on one configuration."""
    m0 = mass + 4.0
    if method == "normal":  # solve_normal(U, D^dag eta), measurements.py:343-346
        b = ctx.apply("DDAG", gauge, mass, eta)
        x, st = ctx.solve(gauge, b, mass, op="normal", tol=tol, maxiter=maxiter, inner=inner)
        return x, st
    if method != "eo":
        raise ValueError(f"unknown propagator method {method!r}")
    even, odd = _parity_masks(ctx.lattice_shape, eta.device)
    b_e, b_o = eta * even, eta * odd
    # rhs_e = b_e - (1/m0) P_e K b_o with K = D - m0 (su3_wilson_nf2.py:1325-1327)
    kbo = ctx.apply("D", gauge, mass, b_o) - m0 * b_o
    rhs_e = b_e - (kbo * even) / m0
    # S_e x_e = rhs_e with S_e = m0 M (M the normalized Schur operator): solve M^dag M x_e = M^dag rhs_e / m0
    rhs_n = ctx.apply("SCHUR_E_DAG", gauge, mass, rhs_e / m0, normalized=True)
    x_e, st = ctx.solve(gauge, rhs_n, mass, op="eo_normal", tol=tol, maxiter=maxiter, inner=inner)
    x_e = x_e * even
    # x_o = (b_o - P_o K x_e) / m0  (su3_wilson_nf2.py:1335)
    kxe = ctx.apply("D", gauge, mass, x_e) - m0 * x_e
    x_o = (b_o - kxe * odd) / m0
    return x_e + x_o, st


def point_source_propagator(theory, U, source: Sequence[int], *, method: str = "normal",
                            tol: Optional[float] = None) -> Tuple[torch.Tensor, Dict[str, float]]:
    """Full point-source propagator S(x)_{s c; s0 c0} for every configuration of U
    (measurements.py:277-372), shape (B, *L, 4, 3, 4, 3) (sink spin, colour,
    source spin, colour), complex128 on the device, plus solver timing/stats."""
    gauges = theory._gauges_for(U)
    shape = tuple(theory.lattice_shape)
    dev = theory.device
    eta = point_sources(shape, source, dev)
    tol = theory.cg_tol if tol is None else float(tol)
    props, stats = [], []
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for g in gauges:
        x, st = propagator_columns(theory.ctx, g, theory.mass, eta, method=method,
                                   inner=theory.solver_precision, tol=tol, maxiter=theory.cg_maxiter)
        stats.extend(st)
        # columns [k = 3 s0 + c0][*L][s][c] -> [*L][s][c][s0][c0]
        props.append(x.reshape(4, 3, *shape, 4, 3).permute(2, 3, 4, 5, 6, 7, 0, 1))
    torch.cuda.synchronize(dev)
    dt = time.perf_counter() - t0
    info = {"inv_n_solves": float(len(stats)), "inv_solve_total_sec_this_call": dt,
            "inv_used_normal_equations": 1.0, "inv_iters_max": float(max(s["iters"] for s in stats)),
            "inv_true_res_max": float(max(s["true_res"] for s in stats)),
            "inv_all_converged": float(all(s["status"] == L.SLOT_CONVERGED for s in stats))}
    return torch.stack(props), info


def pion_two_point(ctx: L.WilsonContext, prop: torch.Tensor, source_t: int) -> np.ndarray:
    """C_pi(dt) = sum_x tr[S(x, 0) S(x, 0)^dag] over the timeslice source_t + dt, summed
    over the batch (measurements.py:375-390).  prop: (B, *L, 4, 3, 4, 3) or columns (n, *L, 4, 3)."""
    shape = tuple(ctx.lattice_shape)
    if prop.dim() == 9:  # (B, *L, s, c, s0, c0) -> columns (B*12, *L, s, c)
        prop = prop.permute(0, 7, 8, 1, 2, 3, 4, 5, 6).reshape(-1, *shape, 4, 3)
    return ctx.pion_correlator(prop.contiguous(), source_t)
