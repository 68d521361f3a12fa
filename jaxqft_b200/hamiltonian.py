"""Monomial protocol and Hamiltonian sum, mirroring ``jaxqft/core/hamiltonian.py``."""

# Portions of this file are transcribed from jaxqft/core/hamiltonian.py of jaxQFT
# (https://github.com/orginos/jaxQFT), under the following license:
#
# BSD 3-Clause License
#
# Copyright (c) 2026, Kostas Orginos
#
# Redistribution and use in source and binary forms, with or without
# modification, are permitted provided that the following conditions are met:
#
# 1. Redistributions of source code must retain the above copyright notice, this
#    list of conditions and the following disclaimer.
#
# 2. Redistributions in binary form must reproduce the above copyright notice,
#    this list of conditions and the following disclaimer in the documentation
#    and/or other materials provided with the distribution.
#
# 3. Neither the name of the copyright holder nor the names of its
#    contributors may be used to endorse or promote products derived from
#    this software without specific prior written permission.
#
# THIS SOFTWARE IS PROVIDED BY THE COPYRIGHT HOLDERS AND CONTRIBUTORS "AS IS"
# AND ANY EXPRESS OR IMPLIED WARRANTIES, INCLUDING, BUT NOT LIMITED TO, THE
# IMPLIED WARRANTIES OF MERCHANTABILITY AND FITNESS FOR A PARTICULAR PURPOSE ARE
# DISCLAIMED. IN NO EVENT SHALL THE COPYRIGHT HOLDER OR CONTRIBUTORS BE LIABLE
# FOR ANY DIRECT, INDIRECT, INCIDENTAL, SPECIAL, EXEMPLARY, OR CONSEQUENTIAL
# DAMAGES (INCLUDING, BUT NOT LIMITED TO, PROCUREMENT OF SUBSTITUTE GOODS OR
# SERVICES; LOSS OF USE, DATA, OR PROFITS; OR BUSINESS INTERRUPTION) HOWEVER
# CAUSED AND ON ANY THEORY OF LIABILITY, WHETHER IN CONTRACT, STRICT LIABILITY,
# OR TORT (INCLUDING NEGLIGENCE OR OTHERWISE) ARISING IN ANY WAY OUT OF THE USE
# OF THIS SOFTWARE, EVEN IF ADVISED OF THE POSSIBILITY OF SUCH DAMAGE.
#
# The Monomial protocol and HamiltonianModel are transcribed method for method (the drop-in keeps
# this interface unchanged); only the JAX typing is removed.

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
