"""SU(3) gauge + Nf=2 Wilson fermions on B200: the drop-in for
``jaxqft/models/su3_wilson_nf2.py``.

``SU3WilsonNf2`` keeps the reference's configuration fields, method names,
argument meaning and array layouts (links ``[B, 4, Lx, Ly, Lz, Lt, 3, 3]``,
fermions ``[B, Lx, Ly, Lz, Lt, 4, 3]``), and runs every fermion operation
through the sm_100a library (``jaxqft_b200.lib``): D, D^dag, the even/odd
blocks and Schur complements, the CG solves (FP64, or FP32/FP16 iteration with
FP64 reliable updates and an FP64 true-residual stopping rule) and the
pseudofermion force.  Inputs may be torch tensors or numpy arrays; outputs are
CUDA tensors of ``dtype`` (complex128 by default, so the HMC Hamiltonian and
Metropolis step are FP64).  There is no CPU fallback.
"""

from __future__ import annotations

import math
import warnings
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple

import numpy as np
import torch

from . import lib as L
from .gamma import build_euclidean_gamma
from .hamiltonian import HamiltonianModel
from .su3_ym import SU3YangMills, project_su3_algebra
from .wilson import WilsonDiracOperator


def _vdot(a: torch.Tensor, b: torch.Tensor) -> torch.Tensor:
    return (a.conj() * b).sum()


def _field_norm(x: torch.Tensor) -> torch.Tensor:
    return torch.sqrt(_vdot(x, x).real)


class _TensorAlgebra:
    """Inner products and linear combinations of the predictors as plain tensor
    algebra (any torch device; the CPU tests of the predictors use it)."""

    @staticmethod
    def dots(pairs) -> np.ndarray:
        return np.array([complex(_vdot(a, b)) for a, b in pairs], dtype=np.complex128)

    @staticmethod
    def combine(coefs, xs) -> torch.Tensor:
        out = torch.zeros_like(xs[0])
        for c, x in zip(coefs, xs):
            out = out + complex(c) * x
        return out


class _DeviceAlgebra:
    """The same on the library's kernels (wl_field_dots: all inner products of a
    predictor in one launch, one pass per pair; wl_field_combine: a combination
    in one pass)."""

    def __init__(self, ctx: L.WilsonContext):
        self.ctx = ctx

    def dots(self, pairs) -> np.ndarray:
        return self.ctx.field_dots(pairs)

    def combine(self, coefs, xs) -> torch.Tensor:
        return self.ctx.field_combine(coefs, xs)


def _chrono_predict(history: List[torch.Tensor], mode: str, max_hist: int, la=None) -> Optional[torch.Tensor]:
    """Initial-guess extrapolation from previous solutions (su3_wilson_nf2.py:85-111):
    'last' or the uniform-step polynomial sum_j (-1)^j C(p, j+1) x_{k-j}."""
    if not history:
        return None
    la = _TensorAlgebra if la is None else la
    h = history[-max(1, int(max_hist)):]
    if len(h) == 1 or mode == "last":
        return h[-1]
    p = len(h)
    return la.combine([float(((-1) ** j) * math.comb(p, j + 1)) for j in range(p)], [h[-1 - j] for j in range(p)])


# _chrono_predict_mre condenses _chrono_predict_mre of jaxqft/models/su3_wilson_nf2.py:114-194
# (jaxQFT, BSD 3-Clause License, Copyright (c) 2026, Kostas Orginos; the full notice is in
# jaxqft_b200/update.py): its damping, regularisation and safeguard steps and constants are the
# reference's, since the predictor must reproduce the reference's initial guesses.
def _chrono_predict_mre(xs: List[torch.Tensor], ys: List[torch.Tensor], target: torch.Tensor,
                        reg: float = 1e-12, la=None) -> Optional[torch.Tensor]:
    """Minimal-residual extrapolation (su3_wilson_nf2.py:114-194): with history
    pairs (x_i, y_i = L x_i), minimise ||target - sum_i c_i y_i|| over c with
    older entries damped by exp(-0.35 age), Tikhonov regularisation reg*tr(G)/n,
    and the reference's safeguards (coefficient bounds, trust-region blend
    towards x_last, norm growth limit, and acceptance only if the subspace
    residual beats the latest image by 3 %).  Inner products and combinations
    run through `la` (the device kernels in the theory); the n x n solve on the
    host, as in the reference."""
    if not xs or not ys:
        return None
    if len(xs) == 1:
        return xs[-1]
    la = _TensorAlgebra if la is None else la
    n = len(xs)
    w = np.asarray([math.exp(-0.35 * float((n - 1) - i)) for i in range(n)])
    upper = [(i, j) for i in range(n) for j in range(i, n)]
    d = la.dots([(ys[i], target) for i in range(n)] + [(ys[i], ys[j]) for i, j in upper])
    g = w * d[:n]
    G = np.zeros((n, n), dtype=np.complex128)
    for (i, j), v in zip(upper, d[n:]):
        G[i, j] = w[i] * w[j] * v
        G[j, i] = np.conj(G[i, j])
    lam = float(reg) * max(1.0, abs(float(np.trace(G).real)) / max(1, n))
    Greg = G + lam * np.eye(n, dtype=np.complex128)
    try:
        c = np.linalg.solve(Greg, g)
    except np.linalg.LinAlgError:
        c, *_ = np.linalg.lstsq(Greg, g, rcond=None)
    c = c * w
    if not np.all(np.isfinite(c)):
        return xs[-1]
    cmax, cl1 = float(np.max(np.abs(c))), float(np.sum(np.abs(c)))
    if cmax > 2.0 or cl1 > 3.0:
        return xs[-1]
    # x0 = beta sum_i c_i x_i + (1 - beta) x_last, in one combination
    beta = 1.0 / max(1.0, cl1)
    cx = beta * c
    cx[-1] += 1.0 - beta
    x0 = la.combine(list(cx), xs)
    # target - sum_i c_i y_i and target - y_last
    r_comb = la.combine([1.0] + list(-c), [target] + list(ys))
    r_last = la.combine([1.0, -1.0], [target, ys[-1]])
    nn = la.dots([(xs[-1], xs[-1]), (x0, x0), (r_comb, r_comb), (r_last, r_last)]).real
    n_last, n_x0, r_mre, r_lst = (math.sqrt(max(v, 0.0)) if math.isfinite(v) else float("nan") for v in nn)
    if not math.isfinite(n_x0) or (n_last > 0.0 and n_x0 > 5.0 * n_last):
        return xs[-1]
    if not (math.isfinite(r_mre) and math.isfinite(r_lst)) or r_mre >= 0.97 * r_lst:
        return xs[-1]
    return x0


@dataclass
class GaugeActionMonomial:
    """Plaquette monomial (su3_wilson_nf2.py:197-214)."""

    model: "SU3WilsonNf2"
    name: str = "gauge"
    timescale: int = 0
    stochastic: bool = False

    def refresh(self, q, traj_length: float = 1.0) -> None:
        return None

    def action(self, q):
        return SU3YangMills.action(self.model, q)

    def force(self, q):
        return SU3YangMills.force(self.model, q)


@dataclass
class _PFBase:
    model: "SU3WilsonNf2"
    name: str = "wilson_nf2_pf"
    timescale: int = 1
    stochastic: bool = True
    refresh_mode: str = "heatbath"
    gamma: float = 0.3
    force_mode: str = "analytic"
    eta: Optional[torch.Tensor] = field(default=None, init=False, repr=False)
    phi: Optional[torch.Tensor] = field(default=None, init=False, repr=False)
    _hist: List[torch.Tensor] = field(default_factory=list, init=False, repr=False)
    _img: List[Optional[torch.Tensor]] = field(default_factory=list, init=False, repr=False)

    def clear(self) -> None:
        self.eta = None
        self.phi = None
        self._hist = []
        self._img = []

    def clear_solver_guess(self) -> None:
        self._hist = []
        self._img = []

    def _guess(self):
        """Initial guess from the solve history (su3_wilson_nf2.py:254-284)."""
        m = self.model
        if not m.use_solver_guess:
            return None
        keep = max(1, int(m.solver_guess_history))
        mode = str(m.solver_guess_mode).lower()
        if mode == "mre" and self.eta is not None:
            pairs = [(x, y) for x, y in zip(self._hist[-keep:], self._img[-keep:])
                     if y is not None and y.shape == self.eta.shape]
            if pairs:
                x0 = _chrono_predict_mre([p[0] for p in pairs], [p[1] for p in pairs], self.eta,
                                         la=_DeviceAlgebra(m.ctx))
                if x0 is not None:
                    return x0
            mode = "poly"  # no images / no eta (OU refresh): polynomial fallback
        return _chrono_predict(self._hist, "poly" if mode == "poly" else "last", keep, la=_DeviceAlgebra(m.ctx))

    def _remember(self, x, y=None):
        if self.model.use_solver_guess:
            keep = max(1, int(self.model.solver_guess_history))
            self._hist = (self._hist + [x])[-keep:]
            self._img = (self._img + [y])[-keep:]

    def _ou_coeffs(self, traj_length):
        c1 = math.exp(-float(self.gamma) * float(traj_length))
        return c1, math.sqrt(max(0.0, 1.0 - c1 * c1))

    def force(self, q):
        if self.phi is None:
            self.refresh(q, traj_length=1.0)
        if str(self.force_mode).lower() not in ("analytic", "autodiff"):
            raise ValueError(f"Unknown pseudofermion force mode: {self.force_mode}")
        # the analytic force is the derivative of the action (the reference's
        # own test su3_wilson_nf2.py:2119-2300 checks it against autodiff)
        return self.force_analytic(q, self.phi)


@dataclass
class WilsonNf2PseudofermionMonomial(_PFBase):
    """S_pf = phi^dag (D^dag D)^-1 phi (su3_wilson_nf2.py:217-403)."""

    def refresh(self, q, traj_length: float = 1.0) -> None:
        m = self.model
        mode = str(self.refresh_mode).lower()
        if mode == "heatbath":
            self.eta = m.random_fermion()
            self.phi = m.apply_Ddag(q, self.eta)  # phi = D^dag eta (:296-302)
        elif mode == "ou":
            noise = m.apply_Ddag(q, m.random_fermion())
            c1, c2 = self._ou_coeffs(traj_length)
            self.phi = noise if self.phi is None else c1 * self.phi + c2 * noise
            self.eta = None
        else:
            raise ValueError(f"Unknown pseudofermion refresh mode: {self.refresh_mode}")
        self._hist = []
        self._img = []

    def action(self, q):
        if self.phi is None:
            self.refresh(q, traj_length=1.0)
        return self.model.pseudofermion_action(q, self.phi, tol=self.model.action_cg_tol)

    def force_analytic(self, q, phi):
        m = self.model
        if m.solver_form != "normal":  # D^dag Y = phi, D X = Y (:360-362)
            x, y = m.solve_split_with_intermediate(q, phi)
            return m.pseudofermion_force_from_solution(q, x, y)
        x0 = self._guess()
        x = m.solve_normal(q, phi) if x0 is None else m.solve_normal_with_guess(q, phi, x0)
        y = m.apply_D(q, x)
        self._remember(x, y)
        return m.pseudofermion_force_from_solution(q, x, y)


@dataclass
class WilsonNf2EOPreconditionedMonomial(_PFBase):
    """S_pf = phi_e^dag (M^dag M)^-1 phi_e, M = normalized even Schur operator
    (su3_wilson_nf2.py:406-590)."""

    name: str = "wilson_nf2_eop_pf"

    def refresh(self, q, traj_length: float = 1.0) -> None:
        m = self.model
        mode = str(self.refresh_mode).lower()
        if mode == "heatbath":
            self.eta = m._project_even(m.random_fermion())
            self.phi = m._project_even(m.apply_eo_schur_even_dagger(q, self.eta, normalized=True))
        elif mode == "ou":
            noise = m.apply_eo_schur_even_dagger(q, m._project_even(m.random_fermion()), normalized=True)
            c1, c2 = self._ou_coeffs(traj_length)
            self.phi = noise if self.phi is None else c1 * self.phi + c2 * noise
            self.phi = m._project_even(self.phi)
            self.eta = None
        else:
            raise ValueError(f"Unknown pseudofermion refresh mode: {self.refresh_mode}")
        self._hist = []
        self._img = []

    def action(self, q):
        if self.phi is None:
            self.refresh(q, traj_length=1.0)
        return self.model.eop_pseudofermion_action(q, self.phi, tol=self.model.action_cg_tol)

    def force_analytic(self, q, phi):
        m = self.model
        if m.solver_form != "normal":  # M^dag Y_e = phi_e, M X_e = Y_e (:563-564)
            xe, ye = m.solve_eop_even_split_with_intermediate(q, phi)
            return m.eop_pseudofermion_force_from_solution(q, xe, ye)
        x0 = self._guess()
        xe = m.solve_eop_even_normal(q, phi) if x0 is None else m.solve_eop_even_normal_with_guess(q, phi, x0)
        ye = m.apply_eo_schur_even(q, xe, normalized=True)
        self._remember(xe, ye)
        return m.eop_pseudofermion_force_from_solution(q, xe, ye)


@dataclass
class SU3WilsonNf2(SU3YangMills):
    """Configuration fields follow su3_wilson_nf2.py:593-623.  Additions:
    ``solver_precision`` ('double' = plain FP64 CG, 'single'/'half' = FP32/FP16
    iterated operator with FP64 reliable updates) and ``reliable_delta``."""

    mass: float = 0.0
    wilson_r: float = 1.0
    cg_tol: float = 1e-8
    cg_maxiter: int = 500
    solver_kind: str = "cg"
    solver_form: str = "normal"
    preconditioner_kind: str = "none"
    gmres_restart: int = 32
    gmres_solve_method: str = "batched"
    fermion_bc: Optional[Tuple[complex, ...]] = None
    dirac_kernel: str = "optimized"
    eo_use_half_spinor: bool = True
    include_gauge_monomial: bool = True
    include_fermion_monomial: bool = True
    fermion_monomial_kind: str = "unpreconditioned"
    gauge_timescale: int = 0
    fermion_timescale: int = 1
    pseudofermion_refresh: str = "heatbath"
    pseudofermion_gamma: Optional[float] = None
    pseudofermion_force_mode: str = "analytic"
    smd_gamma: float = 0.3
    auto_refresh_pseudofermions: bool = True
    use_solver_guess: bool = False
    solver_guess_mode: str = "last"
    solver_guess_history: int = 1
    jit_dirac_kernels: bool = True
    jit_solvers: bool = True
    solver_precision: str = "double"
    reliable_delta: float = 0.1
    action_cg_tol: Optional[float] = None  # tighter tolerance for the Metropolis action solves
    requires_trajectory_refresh: bool = field(default=False, init=False)
    _skip_next_trajectory_refresh: bool = field(default=False, init=False, repr=False)

    def __post_init__(self):
        super().__post_init__()
        if self.Nd != 4:
            raise ValueError("the SU(3) Wilson path is 4-dimensional")
        self.solver_kind = str(self.solver_kind).lower()
        self.solver_form = str(self.solver_form).lower()
        self.fermion_monomial_kind = str(self.fermion_monomial_kind).lower()
        self.solver_guess_mode = str(self.solver_guess_mode).lower()
        if self.solver_kind not in ("cg", "bicgstab", "gmres"):
            raise ValueError("solver_kind must be one of: cg, bicgstab, gmres")
        if self.solver_form not in ("normal", "split", "eo_split"):
            raise ValueError("solver_form must be one of: normal, split, eo_split")
        if self.solver_form in ("split", "eo_split") and self.solver_kind == "cg":
            raise ValueError("solver_form=split/eo_split requires a non-Hermitian solver (use solver_kind=bicgstab)")
        if self.preconditioner_kind not in ("none", "jacobi"):
            raise ValueError("preconditioner_kind must be one of: none, jacobi")
        if self.solver_guess_mode not in ("last", "poly", "mre"):
            raise ValueError("solver_guess_mode must be one of: last, poly, mre")
        if int(self.solver_guess_history) <= 0:
            raise ValueError("solver_guess_history must be positive")
        if self.fermion_monomial_kind not in ("unpreconditioned", "eo_preconditioned"):
            raise ValueError("fermion_monomial_kind must be one of: unpreconditioned, eo_preconditioned")
        if abs(float(self.wilson_r) - 1.0) > 1e-12:
            raise NotImplementedError("the projector kernels implement the Wilson parameter r = 1")
        if self.solver_precision not in ("double", "single", "half"):
            raise ValueError("solver_precision must be one of: double, single, half")
        if any(v % 2 for v in self.lattice_shape):
            raise ValueError("every lattice extent must be even (even/odd layout)")
        mode = str(self.pseudofermion_refresh).lower()
        if self.pseudofermion_gamma is None:
            self.pseudofermion_gamma = float(self.smd_gamma) if mode == "ou" else 0.3
        self.fermion_bc = self._normalize_fermion_bc(self.fermion_bc)
        # the reference builds the phase tensor in complex64 (su3_wilson_nf2.py:727)
        self._bc_phases = tuple(complex(np.complex64(p)) for p in self.fermion_bc)
        self._m0 = float(self.mass + self.wilson_r * self.Nd)
        self.gamma = build_euclidean_gamma(4, dtype=torch.complex128, device=self.device)
        self.Ns = 4
        # the reference keeps its WilsonDiracOperator as `dirac`; callers read its flop counter
        self.dirac = WilsonDiracOperator(ndim=4, mass=float(self.mass), wilson_r=float(self.wilson_r),
                                         dtype=self.dtype, gamma=self.gamma)
        self.ctx = L.WilsonContext(self.lattice_shape, bc=self._bc_phases, device=self.device)
        even, odd, _ = self.ctx.eo_maps()
        self._cb_even_idx = torch.from_numpy(even.astype(np.int64)).to(self.device)
        self._cb_odd_idx = torch.from_numpy(odd.astype(np.int64)).to(self.device)
        self._n_sites = int(np.prod(self.lattice_shape))
        par = torch.zeros(self.lattice_shape, dtype=torch.int64, device=self.device)
        for ax, n in enumerate(self.lattice_shape):
            shp = [1] * 4
            shp[ax] = n
            par = par + torch.arange(n, device=self.device).reshape(shp)
        self._mask_even = (par % 2 == 0).to(torch.float64)[None, ..., None, None]
        self._mask_odd = 1.0 - self._mask_even
        self._gauges: List[L.Gauge] = []
        self._gauge_key = None
        self.last_solver_stats: List[Dict] = []
        monomials = []
        if self.include_gauge_monomial:
            monomials.append(GaugeActionMonomial(self, timescale=int(self.gauge_timescale)))
        self.fermion_monomial = None
        if self.include_fermion_monomial:
            cls = (WilsonNf2EOPreconditionedMonomial if self.fermion_monomial_kind == "eo_preconditioned"
                   else WilsonNf2PseudofermionMonomial)
            self.fermion_monomial = cls(self, timescale=int(self.fermion_timescale),
                                        refresh_mode=str(self.pseudofermion_refresh),
                                        gamma=float(self.pseudofermion_gamma),
                                        force_mode=str(self.pseudofermion_force_mode))
            monomials.append(self.fermion_monomial)
        self.hamiltonian = HamiltonianModel(tuple(monomials))
        self.requires_trajectory_refresh = any(bool(getattr(m, "stochastic", False)) for m in monomials)

    # ------------------------------------------------------------------ helpers
    def _normalize_fermion_bc(self, bc):
        if bc is None:
            vals = [1.0 + 0.0j] * self.Nd
        elif isinstance(bc, str):
            vals = [complex(t.strip().replace("I", "j").replace("i", "j")) for t in bc.split(",") if t.strip()]
        else:
            vals = [complex(v) for v in bc]
        if len(vals) != self.Nd:
            raise ValueError(f"fermion_bc must have Nd={self.Nd} entries; got {len(vals)}")
        return tuple(vals)

    def _as_tensor(self, x) -> torch.Tensor:
        if isinstance(x, np.ndarray):
            x = torch.from_numpy(np.ascontiguousarray(x))
        return x.to(device=self.device, dtype=torch.complex128).contiguous()

    def _gauges_for(self, U) -> List[L.Gauge]:
        """Per-configuration device copies of U, refreshed only when U changed
        (same tensor storage and version counter -> reuse)."""
        U = self._as_tensor(U) if not (isinstance(U, torch.Tensor) and U.dtype == torch.complex128
                                      and U.is_cuda and U.is_contiguous()) else U
        # identity + version of a tensor we keep alive: storage reuse by a new
        # tensor cannot alias a cached gauge field
        if (self._gauge_key is not None and self._gauge_key[0] is U and self._gauge_key[1] == U._version
                and len(self._gauges) == U.shape[0]):
            return self._gauges
        Ub = self._to_bm(U).contiguous() if self.layout != "BMXYIJ" else U
        for b in range(Ub.shape[0]):
            if b < len(self._gauges):
                self._gauges[b].update(Ub[b])
            else:
                self._gauges.append(self.ctx.gauge(Ub[b]))
        del self._gauges[Ub.shape[0]:]
        self._gauge_key = (U, U._version)
        return self._gauges

    def _out(self, x: torch.Tensor) -> torch.Tensor:
        return x if self.dtype == torch.complex128 else x.to(self.dtype)

    def _apply_raw(self, op: str, U, psi, normalized: bool = False) -> torch.Tensor:
        gauges = self._gauges_for(U)
        psi = self._as_tensor(psi)
        out = torch.empty_like(psi)
        for b in range(psi.shape[0]):
            self.ctx.apply(op, gauges[b], self.mass, psi[b], normalized=normalized, out=out[b])
        return out

    def _apply(self, op: str, U, psi, normalized: bool = False):
        return self._out(self._apply_raw(op, U, psi, normalized))

    # ------------------------------------------------------------------ shapes / EO helpers
    def fermion_shape(self) -> Tuple[int, ...]:
        return (self.Bs, *self.lattice_shape, self.Ns, 3)

    def _project_even(self, psi):
        return self._as_tensor(psi) * self._mask_even.to(torch.complex128)

    def _project_odd(self, psi):
        return self._as_tensor(psi) * self._mask_odd.to(torch.complex128)

    def _pack_even_sites(self, psi):
        psi = self._as_tensor(psi)
        return psi.reshape(psi.shape[0], self._n_sites, 4, 3)[:, self._cb_even_idx]

    def _pack_odd_sites(self, psi):
        psi = self._as_tensor(psi)
        return psi.reshape(psi.shape[0], self._n_sites, 4, 3)[:, self._cb_odd_idx]

    def _unpack_sites(self, psi_c, idx):
        out = torch.zeros((psi_c.shape[0], self._n_sites, 4, 3), dtype=psi_c.dtype, device=psi_c.device)
        out[:, idx] = psi_c
        return out.reshape(psi_c.shape[0], *self.lattice_shape, 4, 3)

    def _unpack_even_sites(self, psi_c):
        return self._unpack_sites(self._as_tensor(psi_c), self._cb_even_idx)

    def _unpack_odd_sites(self, psi_c):
        return self._unpack_sites(self._as_tensor(psi_c), self._cb_odd_idx)

    # ------------------------------------------------------------------ operators (:1036-1155)
    def apply_D(self, U, psi):
        return self._apply("D", U, psi)

    def apply_Ddag(self, U, psi):
        return self._apply("DDAG", U, psi)

    def apply_normal(self, U, psi):
        return self._apply("DDAGD", U, psi)

    def apply_D_with_kernel(self, U, psi, kernel: str = "optimized", use_sparse_gamma: bool = True):
        return self.apply_D(U, psi)

    def apply_normal_with_kernel(self, U, psi, kernel: str = "optimized", use_sparse_gamma: bool = True):
        return self.apply_normal(U, psi)

    apply_D_dense = apply_D
    apply_Ddag_dense = apply_Ddag
    apply_normal_dense = apply_normal

    def apply_offdiag(self, U, psi):
        return self._apply("HOP", U, psi)

    def apply_offdiag_dagger(self, U, psi):
        return self._apply("HOP_DAG", U, psi)

    def apply_K_oe(self, U, psi_even):
        return self._apply("K_OE", U, psi_even)

    def apply_K_eo(self, U, psi_odd):
        return self._apply("K_EO", U, psi_odd)

    def apply_Kdag_oe(self, U, psi_even):
        return self._apply("KDAG_OE", U, psi_even)

    def apply_Kdag_eo(self, U, psi_odd):
        return self._apply("KDAG_EO", U, psi_odd)

    def apply_eo_schur_even(self, U, psi_even, normalized: bool = False):
        return self._apply("SCHUR_E", U, psi_even, normalized)

    def apply_eo_schur_even_dagger(self, U, psi_even, normalized: bool = False):
        return self._apply("SCHUR_E_DAG", U, psi_even, normalized)

    def apply_eo_schur_odd(self, U, psi_odd, normalized: bool = False):
        return self._apply("SCHUR_O", U, psi_odd, normalized)

    def apply_eo_schur_even_compact(self, U, psi_even, daggered: bool = False, normalized: bool = True):
        return self._apply("SCHUR_E_DAG" if daggered else "SCHUR_E", U, psi_even, normalized)

    # ------------------------------------------------------------------ random fields
    def random_fermion(self):
        """Complex Gaussian with E|z|^2 = 1 (su3_wilson_nf2.py:1169-1175), drawn by the
        device generator (wl_random_spinor) with the theory's seed and a fresh stream."""
        return self._out(self.ctx.random_spinor(self.Bs, self.seed, self._next_stream()))

    def sample_pseudofermion(self, U):
        return self.apply_Ddag(U, self.random_fermion())

    # ------------------------------------------------------------------ solves (:1243-1454)
    def _solve(self, op: str, U, rhs, x0=None, tol: Optional[float] = None):
        return self._out(self._solve_raw(op, U, rhs, x0, tol))

    def _solve_raw(self, op: str, U, rhs, x0=None, tol: Optional[float] = None) -> torch.Tensor:
        gauges = self._gauges_for(U)
        tol = self.cg_tol if tol is None else float(tol)
        rhs = self._as_tensor(rhs)
        x0 = None if x0 is None else self._as_tensor(x0)
        out = torch.empty_like(rhs)
        stats = []
        for b in range(rhs.shape[0]):
            x, st = self.ctx.solve(gauges[b], rhs[b], self.mass, op=op, tol=tol, maxiter=self.cg_maxiter,
                                   inner=self.solver_precision, delta=self.reliable_delta,
                                   x0=None if x0 is None else x0[b])
            out[b] = x
            stats.extend(st)
        self.last_solver_stats = stats
        if any(s["status"] == L.SLOT_NAN for s in stats):
            raise L.WilsonError(L.WL_ERR_NAN, "solver produced a non-finite residual")
        if any(s["status"] != L.SLOT_CONVERGED for s in stats):
            warnings.warn(f"CG did not reach tol {tol} within {self.cg_maxiter} iterations", RuntimeWarning)
        return out

    def solve_normal(self, U, phi, tol: Optional[float] = None):
        return self._solve("normal", U, phi, tol=tol)

    def solve_normal_with_guess(self, U, phi, x0):
        return self._solve("normal", U, phi, x0)

    def solve_eop_even_normal(self, U, rhs, tol: Optional[float] = None):
        return self._solve("eo_normal", U, self._project_even(rhs), tol=tol)

    def solve_eop_even_normal_with_guess(self, U, rhs, x0):
        return self._solve("eo_normal", U, self._project_even(rhs), self._project_even(x0))

    # Non-Hermitian solves (:1271-1454).  The reference runs BiCGStab / GMRES on D (or on the
    # Schur operator) and stops at ||b - A x|| <= cg_tol ||b|| (relative, atol 0).  Here every one
    # of them is the batched mixed-precision CG on the normal equations of the same operator
    # (CGNR), held to that same stopping rule:
    #   A^dag y = b  <=>  y = A z with A^dag A z = b: the residual b - A^dag y is the normal
    #     residual of z, which CG bounds by cg_tol, so the rule holds as it is;
    #   A x = b  <=>  A^dag A x = A^dag b: CG bounds ||A^dag (b - A x)|| only, so x is refined by
    #     defect correction (_refine_direct) until the FP64 residual ||b - A x|| meets the rule.
    # ``solver_kind`` bicgstab / gmres and ``gmres_restart`` are accepted for configuration
    # compatibility and select the same solver.
    max_refine_rounds = 8  # defect-correction rounds of a direct solve (a class constant)

    def _refine_direct(self, apply_A, solve_normal_eq, b: torch.Tensor, tol: Optional[float]) -> torch.Tensor:
        """x with ||b - A x|| <= tol ||b|| for every batch entry.  solve_normal_eq(r) returns
        the CGNR solution of A x = r; each round solves for the current FP64 residual and adds
        the correction, which shrinks the residual by about cond(A) * tol."""
        tol = self.cg_tol if tol is None else float(tol)
        x = solve_normal_eq(b)
        bn = torch.stack([_field_norm(b[i]) for i in range(b.shape[0])])
        shape = (b.shape[0],) + (1,) * (b.dim() - 1)
        for _ in range(int(self.max_refine_rounds)):
            r = b - apply_A(x)
            rn = torch.stack([_field_norm(r[i]) for i in range(r.shape[0])])
            done = rn <= tol * bn
            if bool(torch.all(done)):
                return x
            # each correction is solved for the residual scaled to unit norm (entries that already
            # meet the rule get a zero right-hand side), so that the reduced-precision iterations
            # see O(1) values however small the residual has become
            scale = torch.where(done, torch.zeros_like(rn), rn)
            inv = torch.where(done, torch.zeros_like(rn), 1.0 / torch.where(done, torch.ones_like(rn), rn))
            x = x + scale.reshape(shape).to(x.dtype) * solve_normal_eq(r * inv.reshape(shape).to(r.dtype))
        warnings.warn(f"direct residual did not reach tol {tol} in {self.max_refine_rounds} refinements",
                      RuntimeWarning)
        return x

    def solve_direct(self, U, rhs, tol: Optional[float] = None):
        """x = D^-1 rhs (:1271-1284), ||rhs - D x|| <= cg_tol ||rhs||."""
        b = self._as_tensor(rhs)
        return self._out(self._refine_direct(
            lambda x: self._apply_raw("D", U, x),
            lambda r: self._solve_raw("normal", U, self._apply_raw("DDAG", U, r), tol=tol), b, tol))

    def solve_dagger(self, U, rhs, tol: Optional[float] = None):
        """y = D^-dag rhs (:1286-1299)."""
        return self._out(self._apply_raw("D", U, self._solve_raw("normal", U, rhs, tol=tol)))

    def _solve_eo(self, U, rhs, which: str, tol: Optional[float] = None) -> torch.Tensor:
        """D x = b (which="direct") or D^dag x = b ("dagger") through the even Schur complement
        and odd-site reconstruction (:1301-1336).  With K = A - m0 (A = D or D^dag):
        rhs_e = b_e - P_e K b_o / m0, S x_e = rhs_e with S = m0 M for "direct" and m0 M^dag for
        "dagger" (M the normalized even Schur operator), x_o = (b_o - P_o K x_e) / m0."""
        if which not in ("direct", "dagger"):
            raise ValueError(f"Unknown EO solve kind: {which}")
        op = "D" if which == "direct" else "DDAG"
        m0 = self._m0
        b = self._as_tensor(rhs)
        b_e, b_o = self._project_even(b), self._project_odd(b)
        rhs_e = b_e - self._project_even(self._apply_raw(op, U, b_o) - m0 * b_o) / m0
        if which == "direct":  # M x_e = rhs_e / m0  <=>  M^dag M x_e = M^dag rhs_e / m0
            x_e = self._solve_schur_direct(U, rhs_e / m0, tol)
        else:  # M^dag x_e = rhs_e / m0  <=>  x_e = M (M^dag M)^-1 rhs_e / m0
            z_e = self._project_even(self._solve_raw("eo_normal", U, rhs_e / m0, tol=tol))
            x_e = self._project_even(self._apply_raw("SCHUR_E", U, z_e, normalized=True))
        x_o = (b_o - self._project_odd(self._apply_raw(op, U, x_e) - m0 * x_e)) / m0
        return x_e + x_o

    def solve_direct_eo(self, U, rhs, tol: Optional[float] = None):
        return self._out(self._solve_eo(U, rhs, "direct", tol))

    def solve_dagger_eo(self, U, rhs, tol: Optional[float] = None):
        return self._out(self._solve_eo(U, rhs, "dagger", tol))

    def _solve_schur_direct(self, U, rhs_e, tol: Optional[float]) -> torch.Tensor:
        """x_e with ||rhs_e - M x_e|| <= tol ||rhs_e||, M the normalized even Schur operator
        (the rule of _solve_eo_one and solve_eop_even_direct, scale-free, so it also holds for
        the unnormalized m0 M)."""
        return self._refine_direct(
            lambda x: self._project_even(self._apply_raw("SCHUR_E", U, x, normalized=True)),
            lambda r: self._project_even(self._solve_raw(
                "eo_normal", U, self._apply_raw("SCHUR_E_DAG", U, r, normalized=True), tol=tol)),
            self._project_even(rhs_e), tol)

    def solve_eop_even_direct(self, U, rhs, tol: Optional[float] = None):
        """M x_e = rhs_e, M the normalized even Schur operator (:1338-1350)."""
        return self._out(self._solve_schur_direct(U, self._as_tensor(rhs), tol))

    def solve_eop_even_dagger(self, U, rhs, tol: Optional[float] = None):
        """M^dag y_e = rhs_e (:1352-1364)."""
        z = self._project_even(self._solve_raw("eo_normal", U, self._project_even(rhs), tol=tol))
        return self._out(self._project_even(self._apply_raw("SCHUR_E", U, z, normalized=True)))

    def solve_eop_even_split_with_intermediate(self, U, phi, tol: Optional[float] = None):
        """y = M^-dag phi, x = M^-1 y (:1394-1397).  With y = M z, z = (M^dag M)^-1 phi, the second
        system M^dag M x = M^dag y has the solution x = z, so the pair costs one solve."""
        z = self._project_even(self._solve_raw("eo_normal", U, self._project_even(phi), tol=tol))
        y = self._project_even(self._apply_raw("SCHUR_E", U, z, normalized=True))
        return self._out(z), self._out(y)

    def solve_eop_even_split(self, U, phi):
        return self.solve_eop_even_split_with_intermediate(U, phi)[0]

    def solve_split_with_intermediate(self, U, phi, tol: Optional[float] = None):
        """y = D^-dag phi, x = D^-1 y (:1438-1445).  "split": y = D z with z = (D^dag D)^-1 phi and
        x = z (the second normal system D^dag D x = D^dag y has the solution z), one solve;
        "eo_split": both solves through the even Schur complement."""
        if self.solver_form == "eo_split":
            y = self._solve_eo(U, phi, "dagger", tol)
            return self._out(self._solve_eo(U, y, "direct", tol)), self._out(y)
        z = self._solve_raw("normal", U, phi, tol=tol)
        return self._out(z), self._out(self._apply_raw("D", U, z))

    def solve_split(self, U, phi):
        return self.solve_split_with_intermediate(U, phi)[0]

    def solve_pseudofermion(self, U, phi):
        if self.solver_form == "normal":
            return self.solve_normal(U, phi)
        return self.solve_split(U, phi)

    def solve_eop_even(self, U, phi):
        if self.solver_form == "normal":
            return self.solve_eop_even_normal(U, phi)
        return self.solve_eop_even_split(U, phi)

    def normal_residual_stats(self, U, phi, x) -> Dict[str, float]:
        r = self.apply_normal(U, x) - self._as_tensor(phi)
        phi = self._as_tensor(phi)
        rel = torch.stack([_field_norm(r[b]) / (_field_norm(phi[b]) + 1e-30) for b in range(r.shape[0])])
        absn = torch.stack([_field_norm(r[b]) for b in range(r.shape[0])])
        return {"mean_rel_residual": float(rel.mean()), "max_rel_residual": float(rel.max()),
                "mean_abs_residual": float(absn.mean()), "max_abs_residual": float(absn.max())}

    def solver_info_stats(self, U, phi) -> Dict[str, float]:
        """Per-RHS iteration counts (su3_wilson_nf2.py:1468-1554): the solve of the
        configured form is run and its CG iterations counted -- for "normal" one
        normal-equation solve per configuration; for "split" / "eo_split" stage 1
        A^dag y = phi and stage 2 A x = y (the direct stage including its
        defect-correction rounds), reported as the stage means and their sum.  The
        counts are real (the reference's JAX solvers report none, so its
        iters_known_fraction is 0 there)."""
        phi = self._as_tensor(phi)
        counts: List[List[int]] = []
        orig = self._solve_raw

        def counting(*a, **k):
            out = orig(*a, **k)
            counts.append([int(st["iters"]) for st in self.last_solver_stats])
            return out

        self._solve_raw = counting
        try:
            B = phi.shape[0]
            if self.solver_form == "normal":
                self.solve_normal(U, phi)
                it = np.asarray(counts[-1], dtype=np.float64)
                it1 = it2 = None
            else:
                eo = self.solver_form == "eo_split"
                counts.clear()
                y = self._solve_eo(U, phi, "dagger") if eo else self.solve_dagger(U, phi)
                it1 = np.sum(np.asarray(counts, dtype=np.float64).reshape(len(counts), B), axis=0)
                counts.clear()
                if eo:
                    self._solve_eo(U, y, "direct")
                else:
                    self.solve_direct(U, y)
                it2 = np.sum(np.asarray(counts, dtype=np.float64).reshape(len(counts), B), axis=0)
                it = it1 + it2
        finally:
            del self._solve_raw
        return {"iters_known_fraction": 1.0, "mean_solver_iters": float(it.mean()),
                "max_solver_iters": float(it.max()),
                "mean_solver_iters_stage1": float(it1.mean()) if it1 is not None else float("nan"),
                "mean_solver_iters_stage2": float(it2.mean()) if it2 is not None else float("nan")}

    # ------------------------------------------------------------------ actions (:1183-1208)
    def _split_chi(self, U, phi, eo_prec: bool, tol: Optional[float] = None) -> torch.Tensor:
        """chi with A^dag chi = phi: S_pf = phi^dag (A^dag A)^-1 phi = chi^dag chi (:1190-1197)."""
        if eo_prec:
            z = self._project_even(self._solve_raw("eo_normal", U, self._project_even(phi), tol=tol))
            return self._project_even(self._apply_raw("SCHUR_E", U, z, normalized=True))
        if self.solver_form == "eo_split":
            return self._solve_eo(U, phi, "dagger", tol)
        return self._apply_raw("D", U, self._solve_raw("normal", U, phi, tol=tol))

    def pseudofermion_action(self, U, phi, tol: Optional[float] = None):
        phi = self._as_tensor(phi)
        if self.solver_form == "normal":
            x = self._solve_raw("normal", U, phi, tol=tol)
            return torch.stack([_vdot(phi[b], x[b]).real for b in range(phi.shape[0])])
        chi = self._split_chi(U, phi, False, tol)
        return torch.stack([_vdot(chi[b], chi[b]).real for b in range(chi.shape[0])])

    def eop_pseudofermion_action(self, U, phi, tol: Optional[float] = None):
        phi = self._project_even(phi)
        if self.solver_form == "normal":
            x = self._solve_raw("eo_normal", U, phi, tol=tol)
            return torch.stack([_vdot(phi[b], x[b]).real for b in range(phi.shape[0])])
        chi = self._split_chi(U, phi, True, tol)
        return torch.stack([_vdot(chi[b], chi[b]).real for b in range(chi.shape[0])])

    # ------------------------------------------------------------------ forces (:1556-1597)
    def pseudofermion_force_from_solution(self, U, X, Y):
        gauges = self._gauges_for(U)
        X, Y = self._as_tensor(X), self._as_tensor(Y)
        F = torch.empty((X.shape[0], 4, *self.lattice_shape, 3, 3), dtype=torch.complex128, device=self.device)
        for b in range(X.shape[0]):
            F[b] = self.ctx.pf_force(gauges[b], X[b], Y[b])
        return self._out(self._from_bm(F))

    def eop_pseudofermion_force_from_solution(self, U, X_e, Y_e):
        """f(K_oe X_e, -a Y_e) + f(X_e, -a K^dag_oe Y_e), a = 1/m0^2."""
        gauges = self._gauges_for(U)
        alpha = 1.0 / (self._m0 * self._m0)
        X_e, Y_e = self._as_tensor(X_e), self._as_tensor(Y_e)
        F = torch.empty((X_e.shape[0], 4, *self.lattice_shape, 3, 3), dtype=torch.complex128, device=self.device)
        for b in range(X_e.shape[0]):
            kx = self.ctx.apply("K_OE", gauges[b], self.mass, X_e[b])
            ky = self.ctx.apply("KDAG_OE", gauges[b], self.mass, Y_e[b])
            Fb = self.ctx.pf_force(gauges[b], kx, Y_e[b], coef=-alpha)
            F[b] = self.ctx.pf_force(gauges[b], X_e[b], ky, coef=-alpha, F=Fb)
        return self._out(self._from_bm(F))

    # ------------------------------------------------------------------ HMC hooks (:1599-1635)
    def prepare_trajectory(self, U, traj_length: float = 1.0) -> None:
        if self._skip_next_trajectory_refresh:
            self._skip_next_trajectory_refresh = False
            return
        self.hamiltonian.prepare_trajectory(U, traj_length=float(traj_length))

    def set_loaded_pseudofermion(self, phi, *, skip_next_refresh: bool = True) -> None:
        if self.fermion_monomial is None:
            raise ValueError("No fermion monomial present; cannot set pseudofermion field")
        self.fermion_monomial.phi = self._as_tensor(phi)
        self.fermion_monomial.eta = None
        self.fermion_monomial.clear_solver_guess()
        if skip_next_refresh:
            self._skip_next_trajectory_refresh = True

    def clear_pseudofermion(self) -> None:
        if self.fermion_monomial is not None:
            self.fermion_monomial.clear()

    def _auto_refresh(self, U):
        if self.auto_refresh_pseudofermions and self.fermion_monomial is not None and self.fermion_monomial.phi is None:
            self.fermion_monomial.refresh(U)

    def action_breakdown(self, U) -> Dict[str, torch.Tensor]:
        self._auto_refresh(U)
        return self.hamiltonian.action_breakdown(U)

    def action(self, U):
        self._auto_refresh(U)
        return self.hamiltonian.action_from_monomials(U)

    def force(self, U):
        self._auto_refresh(U)
        return self.hamiltonian.force_from_monomials(U)

    def gauge_action(self, U):
        return SU3YangMills.action(self, U)

    def gauge_force(self, U):
        return SU3YangMills.force(self, U)
