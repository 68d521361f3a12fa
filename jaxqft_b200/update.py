"""HMC with Metropolis accept/reject, mirroring ``jaxqft/core/update.py:13-126``
(the Python-loop path that theories with a trajectory refresh take)."""

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
