"""HMC with Metropolis accept/reject, mirroring ``jaxqft/core/update.py:13-126``
(the Python-loop path that theories with a trajectory refresh take)."""

# Portions of this file are transcribed from jaxqft/core/update.py of jaxQFT
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
# The Python-loop HMC sequence (refresh, integrate, Metropolis) is kept as the reference runs it.

from __future__ import annotations

from dataclasses import dataclass, field
from typing import Callable, List, Optional

import numpy as np
import torch


@dataclass
class HMC:
    T: object
    I: object
    verbose: bool = True
    seed: int = 0
    AcceptReject: List[float] = field(default_factory=list)
    history: List[dict] = field(default_factory=list)
    uniform: Optional[Callable] = None  # shape -> uniforms in [0,1); default: seeded torch RNG

    def __post_init__(self):
        dev = getattr(self.T, "device", None)
        self.generator = torch.Generator(device=dev if dev is not None else "cpu")
        self.generator.manual_seed(int(self.seed))

    def calc_acceptance(self) -> float:
        return float(np.mean(self.AcceptReject)) if self.AcceptReject else 0.0

    def reset_acceptance(self) -> None:
        self.AcceptReject = []

    def _prepare_trajectory(self, q) -> None:
        if not bool(getattr(self.T, "requires_trajectory_refresh", False)):
            return
        fn = getattr(self.T, "prepare_trajectory", None)
        if not callable(fn):
            raise AttributeError("Theory declares requires_trajectory_refresh=True but has no prepare_trajectory")
        fn(q, traj_length=float(getattr(self.I, "t", 1.0)))

    def evolve(self, q, N: int):
        """N trajectories: refresh, H0, integrate, Hf, Metropolis with exp(-dH)
        in FP64 (update.py:51-78)."""
        for k in range(int(N)):
            self._prepare_trajectory(q)
            q0 = q
            p0 = self.T.refreshP()
            H0 = self.T.kinetic(p0) + self.T.action(q0)
            p, q_prop = self.I.integrate(p0, q0)
            Hf = self.T.kinetic(p) + self.T.action(q_prop)
            dH = (Hf - H0).to(torch.float64)
            acc_prob = torch.where(dH < 0, torch.ones_like(dH), torch.exp(-dH))
            if self.uniform is not None:
                R = torch.as_tensor(self.uniform(acc_prob.shape), dtype=torch.float64, device=acc_prob.device)
            else:
                R = torch.rand(acc_prob.shape, generator=self.generator, device=acc_prob.device, dtype=torch.float64)
            acc = R < acc_prob
            self.AcceptReject.extend(acc.to(torch.float64).cpu().tolist())
            shape = [q.shape[0]] + [1] * (q.ndim - 1)
            q = torch.where(acc.reshape(shape), q_prop, q0)
            self.history.append({"dH": dH.cpu().tolist(), "accepted": acc.cpu().tolist(),
                                 "H0": H0.cpu().tolist()})
            if self.verbose:
                print(" HMC:", k, " dH=", dH.cpu().tolist(), " A/R=", acc.cpu().tolist(),
                      " Pacc=", float(acc.to(torch.float64).mean()))
        return q

    calc_Acceptance = calc_acceptance
    reset_Acceptance = reset_acceptance


hmc = HMC
