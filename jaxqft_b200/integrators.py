"""Molecular-dynamics integrators, mirroring ``jaxqft/core/integrators.py``
(the same update sequences and coefficients, on torch tensors)."""

# Portions of this file are transcribed from jaxqft/core/integrators.py of jaxQFT
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
# The integrators keep the published update sequences and coefficients of the reference
# (leapfrog, MinNorm2 with lambda = 0.1931833275037836, force gradient, MinNorm4PF4).

from __future__ import annotations

from typing import Callable, Tuple


def simple_evolve_p(dt: float, F, P):
    return P + dt * F


class Integrator:
    def __init__(self, force: Callable, evolve_q: Callable, Nmd: int, t: float, evolve_p: Callable = simple_evolve_p):
        self.force, self.evolve_q, self.evolve_p = force, evolve_q, evolve_p
        self.Nmd = int(Nmd)
        self.t = float(t)
        self.dt = self.t / self.Nmd

    def integrate(self, p, q) -> Tuple:
        raise NotImplementedError


class Leapfrog(Integrator):
    """integrators.py:33-43."""

    def integrate(self, p, q):
        p = self.evolve_p(0.5 * self.dt, self.force(q), p)
        for _ in range(1, self.Nmd):
            q = self.evolve_q(self.dt, p, q)
            p = self.evolve_p(self.dt, self.force(q), p)
        q = self.evolve_q(self.dt, p, q)
        p = self.evolve_p(0.5 * self.dt, self.force(q), p)
        return p, q


class MinNorm2(Integrator):
    """Omelyan 2nd order, lambda = 0.1931833275037836 (integrators.py:46-58)."""

    def __init__(self, force, evolve_q, Nmd, t, evolve_p=simple_evolve_p, lam=0.1931833275037836):
        super().__init__(force, evolve_q, Nmd, t, evolve_p)
        self.lam = float(lam)

    def integrate(self, p, q):
        for _ in range(self.Nmd):
            p = self.evolve_p(self.dt * self.lam, self.force(q), p)
            q = self.evolve_q(0.5 * self.dt, p, q)
            p = self.evolve_p(self.dt * (1.0 - 2.0 * self.lam), self.force(q), p)
            q = self.evolve_q(0.5 * self.dt, p, q)
            p = self.evolve_p(self.dt * self.lam, self.force(q), p)
        return p, q


class ForceGradient(Integrator):
    """Chroma-style force-gradient integrator (integrators.py:61-99)."""

    def __init__(self, force, evolve_q, Nmd, t, evolve_p=simple_evolve_p, lam=1.0 / 6.0, xi=1.0 / 72.0):
        super().__init__(force, evolve_q, Nmd, t, evolve_p)
        self.lam, self.xi = float(lam), float(xi)

    def _fg_update(self, p, q, dt1, dt2):
        p_tmp = self.evolve_p(dt1, self.force(q), p * 0)
        q_tmp = self.evolve_q(1.0, p_tmp, q)
        return self.evolve_p(dt2, self.force(q_tmp), p), q

    def integrate(self, p, q):
        dt = self.dt
        lambda_dt = dt * self.lam
        half = 0.5 * dt
        one_m2l = (1.0 - 2.0 * self.lam) * dt
        xi_dtdt = (2.0 * dt * dt * dt * self.xi) / one_m2l
        p = self.evolve_p(lambda_dt, self.force(q), p)
        for _ in range(1, self.Nmd):
            q = self.evolve_q(half, p, q)
            p, q = self._fg_update(p, q, xi_dtdt, one_m2l)
            q = self.evolve_q(half, p, q)
            p = self.evolve_p(2.0 * lambda_dt, self.force(q), p)
        q = self.evolve_q(half, p, q)
        p, q = self._fg_update(p, q, xi_dtdt, one_m2l)
        q = self.evolve_q(half, p, q)
        p = self.evolve_p(lambda_dt, self.force(q), p)
        return p, q


class MinNorm4PF4(Integrator):
    """4th-order minimum-norm integrator (integrators.py:102-129)."""

    def __init__(self, force, evolve_q, Nmd, t, evolve_p=simple_evolve_p, rho=0.1786178958448091,
                 theta=-0.06626458266981843, lam=0.7123418310626056):
        super().__init__(force, evolve_q, Nmd, t, evolve_p)
        self.rho, self.the, self.lam = float(rho), float(theta), float(lam)

    def integrate(self, p, q):
        for _ in range(self.Nmd):
            p = self.evolve_p(self.dt * self.rho, self.force(q), p)
            q = self.evolve_q(self.dt * self.lam, p, q)
            p = self.evolve_p(self.dt * self.the, self.force(q), p)
            q = self.evolve_q(self.dt * (1.0 - 2.0 * self.lam) / 2.0, p, q)
            p = self.evolve_p(self.dt * (1.0 - 2.0 * (self.the + self.rho)), self.force(q), p)
            q = self.evolve_q(self.dt * (1.0 - 2.0 * self.lam) / 2.0, p, q)
            p = self.evolve_p(self.dt * self.the, self.force(q), p)
            q = self.evolve_q(self.dt * self.lam, p, q)
            p = self.evolve_p(self.dt * self.rho, self.force(q), p)
        return p, q


leapfrog = Leapfrog
minnorm2 = MinNorm2
force_gradient = ForceGradient
minnorm4pf4 = MinNorm4PF4
