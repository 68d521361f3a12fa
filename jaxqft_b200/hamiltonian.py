"""Monomial protocol and Hamiltonian sum, mirroring ``jaxqft/core/hamiltonian.py``."""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import Dict, List, Protocol, Sequence, runtime_checkable


@runtime_checkable
class Monomial(Protocol):
    """One Hamiltonian contribution S_i(U) (hamiltonian.py:15-29)."""

    name: str
    timescale: int
    stochastic: bool

    def refresh(self, q, traj_length: float = 1.0) -> None: ...

    def action(self, q): ...

    def force(self, q): ...


@dataclass
class HamiltonianModel:
    """Sum of monomials (hamiltonian.py:32-74)."""

    monomials: Sequence[Monomial] = field(default_factory=tuple)

    def set_monomials(self, monomials: Sequence[Monomial]) -> None:
        self.monomials = tuple(monomials)

    def prepare_trajectory(self, q, traj_length: float = 1.0) -> None:
        for m in self.monomials:
            m.refresh(q, traj_length=float(traj_length))

    def action_from_monomials(self, q):
        if not self.monomials:
            raise ValueError("No monomials configured")
        total = None
        for m in self.monomials:
            term = m.action(q)
            total = term if total is None else total + term
        return total

    def force_from_monomials(self, q):
        if not self.monomials:
            raise ValueError("No monomials configured")
        total = None
        for m in self.monomials:
            term = m.force(q)
            total = term if total is None else total + term
        return total

    def action_breakdown(self, q) -> Dict[str, object]:
        return {m.name: m.action(q) for m in self.monomials}

    def monomial_names(self) -> List[str]:
        return [m.name for m in self.monomials]

    def monomials_by_timescale(self) -> Dict[int, List[Monomial]]:
        out: Dict[int, List[Monomial]] = {}
        for m in self.monomials:
            out.setdefault(int(getattr(m, "timescale", 0)), []).append(m)
        return out
