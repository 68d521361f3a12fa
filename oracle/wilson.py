"""Numpy complex128 restatement of jaxQFT's SU(3) Wilson-fermion path.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).  Array conventions are
the reference's: links ``U[B, mu, Lx, Ly, Lz, Lt, 3, 3]`` (layout BMXYIJ),
spinors ``psi[B, Lx, Ly, Lz, Lt, Ns=4, Nc=3]``; the site flat index is the
C-order ravel of (Lx, Ly, Lz, Lt), so t is fastest.  Each function cites the
reference lines it restates.
"""

from __future__ import annotations

import numpy as np

ND = 4


# --------------------------------------------------------------------------
# gamma algebra (jaxqft/fermions/gamma.py:14-57)
# --------------------------------------------------------------------------
def gamma_matrices() -> np.ndarray:
    """Euclidean Hermitian gammas for Nd=4 by the recursive Kronecker recipe
    of gamma.py:14-46: start from (s1, s2), then (s1 x g for g) + (s2 x I, s3 x I)."""
    s1 = np.array([[0, 1], [1, 0]], dtype=np.complex128)
    s2 = np.array([[0, -1j], [1j, 0]], dtype=np.complex128)
    s3 = np.array([[1, 0], [0, -1]], dtype=np.complex128)
    gam = [s1, s2]
    eye = np.eye(2, dtype=np.complex128)
    gam = [np.kron(s1, g) for g in gam] + [np.kron(s2, eye), np.kron(s3, eye)]
    return np.asarray(gam)


def gamma5(gam: np.ndarray) -> np.ndarray:
    """gamma.py:49-57: i^(d/2) g0 g1 g2 g3."""
    out = (1j) ** (gam.shape[0] // 2) * gam[0]
    for mu in range(1, gam.shape[0]):
        out = out @ gam[mu]
    return out


GAMMA = gamma_matrices()
GAMMA5 = gamma5(GAMMA)


def spin_mul(g: np.ndarray, psi: np.ndarray) -> np.ndarray:
    return np.einsum("st,...tc->...sc", g, psi)


def color_mul(U: np.ndarray, psi: np.ndarray) -> np.ndarray:
    """(U psi)_a = sum_b U_ab psi_b per spin row (wilson.py:107-127)."""
    return np.einsum("...ab,...sb->...sa", U, psi)


def dagger(x: np.ndarray) -> np.ndarray:
    return np.conj(np.swapaxes(x, -1, -2))


# --------------------------------------------------------------------------
# boundary phases (su3_wilson_nf2.py:726-759)
# --------------------------------------------------------------------------
def links_with_bc(U: np.ndarray, bc) -> np.ndarray:
    """Multiply U_mu(x) by bc[mu] on the last slice x_mu = L_mu - 1.  The
    reference builds the phase factor in complex64 (line 727) before casting
    to the field dtype, so the phase is rounded through complex64 here too."""
    U = np.array(U, copy=True)
    lat = U.shape[2:6]
    for mu in range(ND):
        p = complex(np.complex64(complex(bc[mu])))
        if abs(p - 1.0) <= 1e-12:
            continue
        sl = [slice(None)] * U.ndim
        sl[1] = mu
        sl[2 + mu] = lat[mu] - 1
        U[tuple(sl)] *= p
    return U


# --------------------------------------------------------------------------
# full-lattice Wilson operator (wilson.py:134-336)
# --------------------------------------------------------------------------
def dslash(Ubc: np.ndarray, psi: np.ndarray, sign: int, r: float = 1.0) -> np.ndarray:
    """Hopping term, wilson.py:228-256 ("reference" kernel):
    -1/2 sum_mu [(r + sign g_mu) U_mu(x) psi(x+mu) + (r - sign g_mu) U_mu^dag(x-mu) psi(x-mu)].
    ``Ubc`` already carries the boundary phases."""
    out = np.zeros_like(psi)
    for mu in range(ND):
        ax = 1 + mu
        Umu = Ubc[:, mu]
        fwd = color_mul(Umu, np.roll(psi, -1, axis=ax))
        Ub = np.roll(Umu, +1, axis=ax)
        bwd = color_mul(dagger(Ub), np.roll(psi, +1, axis=ax))
        fwd = r * fwd + sign * spin_mul(GAMMA[mu], fwd)
        bwd = r * bwd - sign * spin_mul(GAMMA[mu], bwd)
        out -= 0.5 * (fwd + bwd)
    return out


def apply_D(U, psi, mass, bc, r=1.0):
    """D = (m + r Nd) + dslash(sign=-1) on BC-phased links (su3_wilson_nf2.py:1036-1041)."""
    return (mass + r * ND) * psi + dslash(links_with_bc(U, bc), psi, -1, r)


def apply_Ddag(U, psi, mass, bc, r=1.0):
    return (mass + r * ND) * psi + dslash(links_with_bc(U, bc), psi, +1, r)


def apply_normal(U, psi, mass, bc, r=1.0):
    """D^dag D split into two calls (su3_wilson_nf2.py:1101-1105)."""
    return apply_Ddag(U, apply_D(U, psi, mass, bc, r), mass, bc, r)


def apply_hop(U, psi, bc, dag=False, r=1.0):
    """K = D - m0 (apply_offdiag / apply_offdiag_dagger, su3_wilson_nf2.py:1047-1055)."""
    return dslash(links_with_bc(U, bc), psi, +1 if dag else -1, r)


# --------------------------------------------------------------------------
# even/odd geometry (su3_wilson_nf2.py:819-932)
# --------------------------------------------------------------------------
def parity_field(shape) -> np.ndarray:
    par = np.zeros(shape, dtype=np.int64)
    for ax, n in enumerate(shape):
        s = [1] * len(shape)
        s[ax] = n
        par = par + np.arange(n).reshape(s)
    return par % 2


def cb_indices(shape):
    """Even/odd flat index lists in ascending order (831-840)."""
    flat = parity_field(shape).reshape(-1)
    return (np.flatnonzero(flat == 0).astype(np.int32), np.flatnonzero(flat == 1).astype(np.int32))


def shift_flat(shape, flat_idx, mu, step):
    coords = np.array(np.unravel_index(flat_idx, shape), dtype=np.int64)
    coords[mu] = (coords[mu] + step) % shape[mu]
    return np.ravel_multi_index(coords, shape).astype(np.int32)


def cb_neighbor_maps(shape):
    """Compact neighbour tables (847-882).  Returns a dict with keys
    target_oe, plus_oe, minus_oe, bwd_oe and the eo counterparts."""
    even, odd = cb_indices(shape)
    vol = int(np.prod(shape))
    einv = np.full(vol, -1, dtype=np.int32)
    oinv = np.full(vol, -1, dtype=np.int32)
    einv[even] = np.arange(even.size, dtype=np.int32)
    oinv[odd] = np.arange(odd.size, dtype=np.int32)
    m = {k: [] for k in ("plus_oe", "minus_oe", "bwd_oe", "plus_eo", "minus_eo", "bwd_eo")}
    for mu in range(ND):
        op, om = shift_flat(shape, odd, mu, +1), shift_flat(shape, odd, mu, -1)
        m["plus_oe"].append(einv[op])
        m["minus_oe"].append(einv[om])
        m["bwd_oe"].append(om)
        ep, em = shift_flat(shape, even, mu, +1), shift_flat(shape, even, mu, -1)
        m["plus_eo"].append(oinv[ep])
        m["minus_eo"].append(oinv[em])
        m["bwd_eo"].append(em)
    out = {k: np.stack(v, axis=0) for k, v in m.items()}
    out["target_oe"] = odd
    out["target_eo"] = even
    return out


def mask(shape, parity):
    return (parity_field(shape) == parity).astype(np.float64)[None, ..., None, None]


def project(psi, parity):
    return psi * mask(psi.shape[1:5], parity)


def pack(psi, parity):
    """(B, L..., 4, 3) -> (B, Vh, 4, 3) in ascending flat order (894-909)."""
    shape = psi.shape[1:5]
    idx = cb_indices(shape)[parity]
    return psi.reshape(psi.shape[0], -1, 4, 3)[:, idx]


def unpack(psi_c, shape, parity):
    """Inverse of ``pack`` with zeros on the other parity (911-932)."""
    B = psi_c.shape[0]
    idx = cb_indices(shape)[parity]
    out = np.zeros((B, int(np.prod(shape)), 4, 3), dtype=psi_c.dtype)
    out[:, idx] = psi_c
    return out.reshape(B, *shape, 4, 3)


# --------------------------------------------------------------------------
# masked even/odd blocks and Schur complements (1057-1155)
# --------------------------------------------------------------------------
def K_block(U, psi, bc, src_parity, dag=False):
    """K_oe (src even -> odd), K_eo (src odd -> even) and daggers, masked (1057-1099)."""
    return project(apply_hop(U, project(psi, src_parity), bc, dag=dag), 1 - src_parity)


def m0_of(mass, r=1.0):
    return mass + r * ND


def schur_even(U, psi_e, mass, bc, normalized=False, dag=False):
    """S_e = m0 - (1/m0) K_eo K_oe (normalized: divided by m0), 1112-1146."""
    m0 = m0_of(mass)
    xe = project(psi_e, 0)
    z = K_block(U, K_block(U, xe, bc, 0, dag), bc, 1, dag)
    if normalized:
        return xe - z / (m0 * m0)
    return m0 * xe - z / m0


def schur_odd(U, psi_o, mass, bc, normalized=False):
    m0 = m0_of(mass)
    xo = project(psi_o, 1)
    z = K_block(U, K_block(U, xo, bc, 1), bc, 0)
    if normalized:
        return xo - z / (m0 * m0)
    return m0 * xo - z / m0


def compact_hop(Ubc_one, psi_c, shape, sign, target):
    """Compact parity hop for one configuration (934-966), full-projector form.
    ``target`` 'oe' maps compact-even -> compact-odd, 'eo' the reverse."""
    maps = cb_neighbor_maps(shape)
    tgt = maps["target_" + target]
    plus, minus, bwd = maps["plus_" + target], maps["minus_" + target], maps["bwd_" + target]
    out = np.zeros_like(psi_c)
    for mu in range(ND):
        Umu = Ubc_one[mu].reshape(-1, 3, 3)
        Uf = Umu[tgt]
        Ub = dagger(Umu[bwd[mu]])
        f = color_mul(Uf, psi_c[plus[mu]])
        b = color_mul(Ub, psi_c[minus[mu]])
        f = f + sign * spin_mul(GAMMA[mu], f)
        b = b - sign * spin_mul(GAMMA[mu], b)
        out -= 0.5 * (f + b)
    return out


def schur_even_compact(U, psi_e_c, mass, bc, shape, dag=False, normalized=True):
    """Compact-even Schur matvec per configuration (976-988)."""
    m0 = m0_of(mass)
    sign = +1 if dag else -1
    Ubc = links_with_bc(U, bc)
    out = np.empty_like(psi_e_c)
    for b in range(psi_e_c.shape[0]):
        y = compact_hop(Ubc[b], psi_e_c[b], shape, sign, "oe")
        z = compact_hop(Ubc[b], y, shape, sign, "eo")
        out[b] = psi_e_c[b] - z / (m0 * m0) if normalized else m0 * psi_e_c[b] - z / m0
    return out


# --------------------------------------------------------------------------
# CG (JAX's published algorithm, as called by su3_wilson_nf2.py:1243-1269)
# --------------------------------------------------------------------------
def vdot(a, b):
    return np.vdot(np.asarray(a).ravel(), np.asarray(b).ravel())


def cg(A, b, tol, maxiter, x0=None):
    """Textbook CG with JAX's stopping rule ||r||^2 <= tol^2 ||b||^2 (atol=0)."""
    x = np.zeros_like(b) if x0 is None else np.array(x0, copy=True)
    r = b - A(x)
    p = r.copy()
    gamma = vdot(r, r).real
    bs = vdot(b, b).real
    k = 0
    while gamma > tol * tol * bs and k < maxiter:
        Ap = A(p)
        alpha = gamma / vdot(p, Ap).real
        x = x + alpha * p
        r = r - alpha * Ap
        g2 = vdot(r, r).real
        p = r + (g2 / gamma) * p
        gamma = g2
        k += 1
    return x, k


def solve_normal(U, phi, mass, bc, tol, maxiter, x0=None):
    """Per-configuration CG on D^dag D (1410-1432).  Returns (x, iters list)."""
    xs, its = [], []
    for b in range(phi.shape[0]):
        A = lambda v, b=b: apply_normal(U[b:b + 1], v[None], mass, bc)[0]
        x, k = cg(A, phi[b], tol, maxiter, None if x0 is None else x0[b])
        xs.append(x)
        its.append(k)
    return np.stack(xs), its


def solve_eop_even_normal(U, rhs, mass, bc, tol, maxiter, x0=None):
    """CG on M^dag M, M = normalized compact even Schur operator (1370-1392)."""
    shape = rhs.shape[1:5]
    bc_ = pack(project(rhs, 0), 0)
    x0c = None if x0 is None else pack(project(x0, 0), 0)
    xs, its = [], []
    for b in range(rhs.shape[0]):
        def A(v, b=b):
            y = schur_even_compact(U[b:b + 1], v[None], mass, bc, shape, dag=False)
            return schur_even_compact(U[b:b + 1], y, mass, bc, shape, dag=True)[0]

        x, k = cg(A, bc_[b], tol, maxiter, None if x0c is None else x0c[b])
        xs.append(x)
        its.append(k)
    return unpack(np.stack(xs), shape, 0), its


def pseudofermion_action(U, phi, mass, bc, tol, maxiter):
    """S_pf = Re phi^dag (D^dag D)^-1 phi per configuration (1183-1196)."""
    x, _ = solve_normal(U, phi, mass, bc, tol, maxiter)
    return np.array([vdot(phi[b], x[b]).real for b in range(phi.shape[0])])


def eop_pseudofermion_action(U, phi_e, mass, bc, tol, maxiter):
    phi_e = project(phi_e, 0)
    x, _ = solve_eop_even_normal(U, phi_e, mass, bc, tol, maxiter)
    return np.array([vdot(phi_e[b], x[b]).real for b in range(phi_e.shape[0])])


# --------------------------------------------------------------------------
# forces (su3_wilson_nf2.py:1556-1597; su3_ym.py:63-67)
# --------------------------------------------------------------------------
def ta(x):
    """Traceless anti-Hermitian projection, su3_ym.py:63-67."""
    y = 0.5 * (x - dagger(x))
    tr = np.trace(y, axis1=-2, axis2=-1)[..., None, None] / 3.0
    return y - tr * np.eye(3)


def force_from_solution(U, X, Y, bc, r=1.0):
    """Link force from (X, Y), 1556-1576: per mu
    c1 = sum_st conj(Y(x))_sa (r - g)_st (U X(x+mu))_tc,
    c2 = sum conj(Y(x+mu))_sa (r + g)_st U^dag_ad X(x)_tc,
    F_mu = TA(transpose(c1 - c2))."""
    Ubc = links_with_bc(U, bc)
    eye = np.eye(4)
    out = []
    for mu in range(ND):
        ax = 1 + mu
        Umu = Ubc[:, mu]
        UX = color_mul(Umu, np.roll(X, -1, axis=ax))
        Yp = np.roll(Y, -1, axis=ax)
        c1 = np.einsum("...sa,st,...tc->...ac", np.conj(Y), r * eye - GAMMA[mu], UX, optimize=True)
        c2 = np.einsum("...sa,st,...ad,...tc->...dc", np.conj(Yp), r * eye + GAMMA[mu], dagger(Umu), X,
                       optimize=True)
        out.append(ta(np.swapaxes(c1 - c2, -1, -2)))
    return np.stack(out, axis=1)


def eop_force_from_solution(U, Xe, Ye, mass, bc):
    """EO force, 1578-1597: f(K_oe X_e, -a Y_e) + f(X_e, -a K^dag_oe Y_e), a = 1/m0^2."""
    a = 1.0 / m0_of(mass) ** 2
    kx = K_block(U, Xe, bc, 0)
    ky = K_block(U, Ye, bc, 0, dag=True)
    return force_from_solution(U, kx, -a * Ye, bc) + force_from_solution(U, Xe, -a * ky, bc)


# --------------------------------------------------------------------------
# gauge pieces (su3_ym.py:339-388, 252-337)
# --------------------------------------------------------------------------
def plaquette_sum(U):
    """sum_{x, mu<nu} Re Tr U_mu(x) U_nu(x+mu) U_mu(x+nu)^dag U_nu(x)^dag."""
    s = np.zeros(U.shape[0])
    for mu in range(ND):
        for nu in range(mu + 1, ND):
            Um, Un = U[:, mu], U[:, nu]
            p = Um @ np.roll(Un, -1, axis=1 + mu) @ dagger(np.roll(Um, -1, axis=1 + nu)) @ dagger(Un)
            s += np.real(np.trace(p, axis1=-2, axis2=-1)).reshape(U.shape[0], -1).sum(axis=1)
    return s


def gauge_action(U, beta):
    return -(beta / 3.0) * plaquette_sum(U)


def average_plaquette(U):
    vol = int(np.prod(U.shape[2:6]))
    return plaquette_sum(U) / (3.0 * vol * 6)


def gauge_force(U, beta):
    """Left-invariant plaquette force -(beta/3) TA(U_mu staple^dag), su3_ym.py:296-327."""
    out = []
    for mu in range(ND):
        Um = U[:, mu]
        st = np.zeros_like(Um)
        for nu in range(ND):
            if nu == mu:
                continue
            Un = U[:, nu]
            st = st + Un @ np.roll(Um, -1, axis=1 + nu) @ dagger(np.roll(Un, -1, axis=1 + mu))
            Unm = np.roll(Un, +1, axis=1 + nu)
            st = st + dagger(Unm) @ np.roll(Um, +1, axis=1 + nu) @ np.roll(Unm, -1, axis=1 + mu)
        out.append(-(beta / 3.0) * ta(Um @ dagger(st)))
    return np.stack(out, axis=1)


def kinetic(P):
    """-1/2 sum Re Tr P P (su3_ym.py:362-364)."""
    return -0.5 * np.real(np.einsum("...ab,...ba->...", P, P)).reshape(P.shape[0], -1).sum(axis=1)


def expm_su3(X):
    import scipy.linalg as sl

    return sl.expm(X)


def evolve_q(dt, P, U):
    """U <- expm(dt P) U (su3_ym.py:352-355, exp_method='expm')."""
    return expm_su3(dt * P) @ U


# --------------------------------------------------------------------------
# HMC molecular dynamics (core/integrators.py:46-58, core/update.py:51-78)
# --------------------------------------------------------------------------
def total_force(U, phi, mass, bc, beta, tol, eo=False):
    """Gauge force + analytic Nf=2 pseudofermion force (monomial force_analytic,
    su3_wilson_nf2.py:374-389 and 566-579)."""
    F = gauge_force(U, beta)
    if eo:
        xe, _ = solve_eop_even_normal(U, phi, mass, bc, tol, 10000)
        ye = schur_even(U, xe, mass, bc, normalized=True)
        return F + eop_force_from_solution(U, xe, ye, mass, bc)
    x, _ = solve_normal(U, phi, mass, bc, tol, 10000)
    return F + force_from_solution(U, x, apply_D(U, x, mass, bc), bc)


def hamiltonian(U, P, phi, mass, bc, beta, tol, eo=False):
    if eo:
        sf = eop_pseudofermion_action(U, phi, mass, bc, tol, 10000)
    else:
        sf = pseudofermion_action(U, phi, mass, bc, tol, 10000)
    return kinetic(P) + gauge_action(U, beta) + sf


def minnorm2(P, U, force, nmd, tau, lam=0.1931833275037836):
    dt = tau / nmd
    for _ in range(nmd):
        P = P + dt * lam * force(U)
        U = evolve_q(0.5 * dt, P, U)
        P = P + dt * (1.0 - 2.0 * lam) * force(U)
        U = evolve_q(0.5 * dt, P, U)
        P = P + dt * lam * force(U)
    return P, U


# --------------------------------------------------------------------------
# seeded inputs
# --------------------------------------------------------------------------
def hot_links(rng, shape, batch, scale):
    """expm(TA(scale (G1 + i G2))) per link: what hot_start(scale) computes
    (su3_ym.py:238-247, 366-367), drawn from a numpy Generator."""
    lshape = (batch, ND, *shape, 3, 3)
    a = scale * (rng.standard_normal(lshape) + 1j * rng.standard_normal(lshape))
    return expm_su3(ta(a))


def hot_links_eigh(rng, shape, batch, scale):
    """Same distribution as ``hot_links`` with exp(X) = V exp(-i lam) V^dag from
    the eigendecomposition of the Hermitian iX (fast at full lattice volumes)."""
    lshape = (batch, ND, *shape, 3, 3)
    a = scale * (rng.standard_normal(lshape) + 1j * rng.standard_normal(lshape))
    X = ta(a)
    lam, V = np.linalg.eigh(1j * X)
    return np.einsum("...ij,...j,...kj->...ik", V, np.exp(-1j * lam), np.conj(V), optimize=True)


def gaussian_spinor(rng, shape, batch):
    fshape = (batch, *shape, 4, 3)
    return (rng.standard_normal(fshape) + 1j * rng.standard_normal(fshape)) / np.sqrt(2.0)


def algebra_field(rng, shape, batch):
    lshape = (batch, ND, *shape, 3, 3)
    return ta(rng.standard_normal(lshape) + 1j * rng.standard_normal(lshape))


def kappa_to_mass(kappa, r=1.0):
    return 1.0 / (2.0 * kappa) - r * ND


# ----------------------------------------------------------------------------- measurements
def point_source_propagator(U, mass, bc, source, tol=1e-12, maxiter=5000):
    """S[b, x, s, c, s0, c0] = (D^{-1} delta_{source, s0, c0})(x)_{s c}: one
    solve_normal(U, apply_Ddag(U, delta)) per (s0, c0), as the iterative
    backend with the CG solver kind does (jaxqft/core/measurements.py:277-372)."""
    B = U.shape[0]
    shape = U.shape[2:6]
    src = tuple(int(v) % int(n) for v, n in zip(source, shape))
    prop = np.zeros((B, *shape, 4, 3, 4, 3), dtype=np.complex128)
    for s0 in range(4):
        for c0 in range(3):
            rhs = np.zeros((B, *shape, 4, 3), dtype=np.complex128)
            rhs[(slice(None), *src, s0, c0)] = 1.0
            x, _ = solve_normal(U, apply_Ddag(U, rhs, mass, bc), mass, bc, tol, maxiter)
            prop[..., s0, c0] = x
    return prop


def pion_two_point(prop, source_t):
    """C(dt) = sum over the timeslice source_t + dt of |S|^2, all batch, spin and
    colour indices (measurements.py:375-390)."""
    lt = prop.shape[4]
    corr = np.zeros(lt)
    for t in range(lt):
        slab = prop[:, :, :, :, t]
        corr[(t - int(source_t)) % lt] = float(np.real(np.sum(np.conj(slab) * slab)))
    return corr
