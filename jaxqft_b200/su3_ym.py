"""SU(3) pure-gauge pieces on the device, mirroring ``jaxqft/models/su3_ym.py``
-- the gauge monomial, momentum refresh, kinetic term, exponential drift and
link generation that an SU(3) + Wilson-fermion HMC needs next to the fermion
path.  The plaquette action, staple force, exp(dt P) U drift and kinetic term
run as sm_100a kernels of libwilson_sm100 (``wl_gauge_*``); momentum refresh
and link generation use the torch CUDA RNG.

Link layout BMXYIJ ``U[B, mu, Lx, Ly, Lz, Lt, 3, 3]`` (``su3_ym.py:246-249``);
BXYMIJ is accepted and converted at the boundary.  Everything is complex128
by default so that the HMC Hamiltonian and the Metropolis step are FP64.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Optional, Tuple

import numpy as np
import torch


def dagger(x: torch.Tensor) -> torch.Tensor:
    return x.conj().transpose(-1, -2)


def project_su3_algebra(x: torch.Tensor) -> torch.Tensor:
    """Traceless anti-Hermitian part: (x - x^dag)/2 - tr/3 (su3_ym.py:63-67)."""
    y = 0.5 * (x - dagger(x))
    tr = torch.diagonal(y, dim1=-2, dim2=-1).sum(-1) / 3.0
    return y - tr[..., None, None] * torch.eye(3, dtype=y.dtype, device=y.device)


def _trace_re(x: torch.Tensor) -> torch.Tensor:
    return torch.diagonal(x, dim1=-2, dim2=-1).sum(-1).real


@dataclass
class SU3YangMills:
    """Wilson plaquette gauge theory in link coordinates (su3_ym.py:180-431)."""

    lattice_shape: Tuple[int, ...]
    beta: float
    batch_size: int = 1
    layout: str = "BMXYIJ"
    seed: int = 0
    exp_method: str = "expm"
    dtype: torch.dtype = torch.complex128
    device: Optional[str] = None

    _wl: Optional[object] = field(init=False, default=None, repr=False)

    def __post_init__(self):
        self.lattice_shape = tuple(int(v) for v in self.lattice_shape)
        self.Nd = len(self.lattice_shape)
        self.Bs = int(self.batch_size)
        self.layout = {"BM...IJ": "BMXYIJ", "B...MIJ": "BXYMIJ"}.get(self.layout.upper(), self.layout.upper())
        if self.layout not in ("BMXYIJ", "BXYMIJ"):
            raise ValueError("layout must be one of: BMXYIJ, BXYMIJ, BM...IJ, B...MIJ")
        self.exp_method = self.exp_method.lower()
        if self.exp_method not in ("expm", "su3"):
            raise ValueError("exp_method must be one of: expm, su3")
        if not torch.cuda.is_available():
            raise RuntimeError("the B200 Wilson-fermion path requires a CUDA device (no CPU fallback)")
        self.device = torch.device(self.device) if self.device is not None else torch.device(
            "cuda", torch.cuda.current_device())
        self._rng_stream = 0  # draws of the device generator so far (one stream each)
        self.mu_axis = 1 if self.layout == "BMXYIJ" else 1 + self.Nd

    # ------------------------------------------------------------------ layout
    def field_shape(self):
        if self.layout == "BMXYIJ":
            return (self.Bs, self.Nd, *self.lattice_shape, 3, 3)
        return (self.Bs, *self.lattice_shape, self.Nd, 3, 3)

    def _to_bm(self, U: torch.Tensor) -> torch.Tensor:
        """Any accepted layout -> BMXYIJ view/copy."""
        if self.layout == "BMXYIJ":
            return U
        return U.movedim(1 + self.Nd, 1)

    def _from_bm(self, U: torch.Tensor) -> torch.Tensor:
        if self.layout == "BMXYIJ":
            return U
        return U.movedim(1, 1 + self.Nd)

    def _take_mu(self, x, mu):
        return x.select(self.mu_axis, mu)

    # ------------------------------------------------------------------ random fields
    def _next_stream(self) -> int:
        """Stream number of the next device-generator draw: each draw of the
        theory uses a fresh stream of the theory's seed, as the reference splits
        a fresh jax.random key per draw (su3_ym.py:234-236)."""
        self._rng_stream += 1
        return self._rng_stream

    def _sample_algebra(self, scale: float = 1.0) -> torch.Tensor:
        """TA(scale (G1 + i G2)) with Gaussian G (su3_ym.py:238-244), drawn by the
        device generator (wl_random_algebra)."""
        P = self._ctx().random_algebra(self.Bs, self.seed, self._next_stream(), scale)
        return self._from_bm(P).to(self.dtype)

    def algebra_to_links(self, q: torch.Tensor) -> torch.Tensor:
        return torch.linalg.matrix_exp(project_su3_algebra(q))

    def hot_start(self, scale: float = 0.1) -> torch.Tensor:
        """exp(TA(scale (G1 + i G2))) = exp(i scale H) per link (su3_ym.py:366-367)."""
        return self.algebra_to_links(self._sample_algebra(scale))

    def refresh_p(self) -> torch.Tensor:
        return self._sample_algebra(1.0)

    # ------------------------------------------------------------------ gauge action / force
    def _ctx(self):
        """Geometry context of the CUDA library (periodic; the gauge kernels ignore fermion BCs)."""
        if self._wl is None:
            if self.Nd != 4:
                raise NotImplementedError("the gauge kernels are written for Nd = 4")
            from .lib import WilsonContext

            self._wl = WilsonContext(self.lattice_shape, bc=(1, 1, 1, 1), device=self.device)
        return self._wl

    def _plaquette_sum(self, U: torch.Tensor) -> torch.Tensor:
        s = self._ctx().plaquette_sum(self._to_bm(U))
        return torch.as_tensor(s, dtype=torch.float64, device=self.device)

    def action(self, U: torch.Tensor) -> torch.Tensor:
        """S_g = -(beta/3) sum_p Re Tr U_p (su3_ym.py:264-280)."""
        return -(self.beta / 3.0) * self._plaquette_sum(U)

    def force(self, U: torch.Tensor) -> torch.Tensor:
        """-(beta/3) TA(U_mu staple^dag), for P <- P + dt F (su3_ym.py:298-327)."""
        return self._from_bm(self._ctx().gauge_force(self._to_bm(U), self.beta))

    def evolve_q(self, dt: float, P: torch.Tensor, Q: torch.Tensor) -> torch.Tensor:
        """U <- exp(dt P) U (su3_ym.py:349-355, exp_method "expm")."""
        return self._from_bm(self._ctx().gauge_evolve(dt, self._to_bm(P), self._to_bm(Q)))

    def kinetic(self, P: torch.Tensor) -> torch.Tensor:
        """-1/2 sum Re Tr P P (su3_ym.py:362-364)."""
        k = self._ctx().kinetic(self._to_bm(P))
        return torch.as_tensor(k, dtype=torch.float64, device=self.device)

    def average_plaquette(self, U: torch.Tensor) -> torch.Tensor:
        vol = math.prod(self.lattice_shape)
        nplanes = self.Nd * (self.Nd - 1) // 2
        return self._plaquette_sum(U) / (3.0 * vol * nplanes)

    def reunitarize(self, U: torch.Tensor) -> torch.Tensor:
        """Project links back onto SU(3) (Gram-Schmidt rows 0,1; row 2 = conj(row0 x row1)).
        The reference's exact exponential drift keeps links in SU(3) to rounding;
        long FP64 trajectories can call this to remove the accumulated drift."""
        r0 = U[..., 0, :]
        r0 = r0 / torch.linalg.vector_norm(r0, dim=-1, keepdim=True)
        r1 = U[..., 1, :]
        r1 = r1 - (r0.conj() * r1).sum(-1, keepdim=True) * r0
        r1 = r1 / torch.linalg.vector_norm(r1, dim=-1, keepdim=True)
        r2 = torch.linalg.cross(r0, r1).conj()
        return torch.stack((r0, r1, r2), dim=-2)

    refreshP = refresh_p
    evolveQ = evolve_q
    hotStart = hot_start
