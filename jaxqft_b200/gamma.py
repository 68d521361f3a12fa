"""Euclidean gamma matrices, mirroring ``jaxqft/fermions/gamma.py`` (torch).

The CUDA kernels hard-code the rank-2 spin projectors of this basis; these
matrices are for host-side checks and users of the drop-in API.
"""

# Portions of this file are transcribed from jaxqft/fermions/gamma.py of jaxQFT
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
# The recursive Kronecker construction of the Euclidean basis is the reference's (bit-exact
# gamma parity needs the same basis), restated on torch tensors.

from __future__ import annotations

from typing import Dict

import torch


def build_euclidean_gamma(ndim: int, dtype=torch.complex128, device=None) -> torch.Tensor:
    """gamma[mu] with {gamma_mu, gamma_nu} = 2 delta_{mu nu} by the recursive
    Kronecker construction of gamma.py:14-46."""
    d = int(ndim)
    if d < 1:
        raise ValueError("ndim must be >= 1")
    s1 = torch.tensor([[0, 1], [1, 0]], dtype=dtype, device=device)
    s2 = torch.tensor([[0, -1j], [1j, 0]], dtype=dtype, device=device)
    s3 = torch.tensor([[1, 0], [0, -1]], dtype=dtype, device=device)
    if d == 1:
        return torch.ones((1, 1, 1), dtype=dtype, device=device)
    if d == 2:
        return torch.stack([s1, s2])
    gam = [s1, s2]
    cur = 2
    while cur + 1 < d:
        eye = torch.eye(gam[0].shape[0], dtype=dtype, device=device)
        gam = [torch.kron(s1, g) for g in gam] + [torch.kron(s2, eye), torch.kron(s3, eye)]
        cur += 2
    if cur == d:
        return torch.stack(gam)
    n = (d - 1) // 2
    g_last = (1j) ** n * gam[0]
    for mu in range(1, d - 1):
        g_last = g_last @ gam[mu]
    return torch.stack(gam + [g_last])


def gamma5(gam: torch.Tensor) -> torch.Tensor:
    """i^(d/2) g_0 ... g_{d-1} for even d (gamma.py:49-57)."""
    d = int(gam.shape[0])
    if d % 2:
        raise ValueError("gamma5 is defined here only for even ndim")
    out = (1j) ** (d // 2) * gam[0]
    for mu in range(1, d):
        out = out @ gam[mu]
    return out


def check_gamma_algebra(gam: torch.Tensor) -> Dict[str, float]:
    d, n = int(gam.shape[0]), int(gam.shape[-1])
    eye = torch.eye(n, dtype=gam.dtype, device=gam.device)
    max_rel = max_herm = 0.0
    for mu in range(d):
        gm = gam[mu]
        max_herm = max(max_herm, float(torch.linalg.matrix_norm(gm - gm.conj().T)))
        for nu in range(d):
            anti = gm @ gam[nu] + gam[nu] @ gm
            target = 2.0 * eye if mu == nu else torch.zeros_like(eye)
            denom = float(torch.linalg.matrix_norm(target)) + 1e-12
            max_rel = max(max_rel, float(torch.linalg.matrix_norm(anti - target)) / denom)
    return {"max_rel_clifford_error": max_rel, "max_hermiticity_error": max_herm}
