"""``jax.scipy.sparse.linalg.cg`` restated on numpy.

Follows JAX's published conjugate-gradient algorithm (jax/_src/scipy/sparse/
linalg.py, ``_cg_solve``): r0 = b - A x0, p0 = M r0, gamma = Re<r, M r>;
loop while Re<r, r> > max(tol^2 Re<b, b>, atol^2) and k < maxiter:
alpha = gamma / Re<p, A p>, x += alpha p, r -= alpha A p, z = M r,
gamma' = Re<r, z>, p = z + (gamma'/gamma) p.  Returns (x, None) like JAX.
``bicgstab``/``gmres`` are deliberately absent (ImportError), which the
reference handles by setting them to None.
"""

from __future__ import annotations

import numpy as _np

from jax.numpy import asarray as _asarray


def _vdot_real(a, b):
    return float(_np.real(_np.vdot(_np.asarray(a).ravel(), _np.asarray(b).ravel())))


def cg(A, b, x0=None, *, tol=1e-5, atol=0.0, maxiter=None, M=None):
    b = _np.asarray(b)
    if x0 is None:
        x0 = _np.zeros_like(b)
    if maxiter is None:
        maxiter = 10 * b.size
    Mf = (lambda v: v) if M is None else M
    bs = _vdot_real(b, b)
    atol2 = max(tol * tol * bs, atol * atol)
    x = _np.asarray(x0)
    r = b - _np.asarray(A(x))
    z = _np.asarray(Mf(r))
    p = z
    gamma = _vdot_real(r, z)
    k = 0
    while True:
        rs = gamma if M is None else _vdot_real(r, r)
        if not (rs > atol2 and k < maxiter):
            break
        Ap = _np.asarray(A(p))
        alpha = gamma / _vdot_real(p, Ap)
        x = x + alpha * p
        r = r - alpha * Ap
        z = _np.asarray(Mf(r))
        gamma_new = _vdot_real(r, z)
        beta = gamma_new / gamma
        p = z + beta * p
        gamma = gamma_new
        k += 1
    cg.last_num_iters = k
    return _asarray(x), None


cg.last_num_iters = 0
