"""Host-side restatement of the tensor-core FP16 hop (jaxqft_b200/csrc/wl_hop_mma.cuh), no GPU.

The kernel computes one site's hop over 8 RHS as 8 mma.sync m16n8k16 tiles
(2 spin pairs x 4 mu; tile j holds RHS 0-7 of output spin 2j in rows 0-7 and
of spin 2j + 1 in rows 8-15), each lane (g, t) holding colour t of RHS g.
This test rebuilds, in float64, every lane's A words (``mma_rows``), B words
(staged link pairs + ``__byte_perm`` selection) and the per-tile matrices of the
PTX fragment layout of m16n8k16 (A: rows g / g + 8, columns 2t, 2t + 1 and
2t + 8, 2t + 9; B: rows 2t, 2t + 1 and 2t + 8, 2t + 9, column g; D: rows g /
g + 8, columns 2t, 2t + 1), multiplies them, and reads the lanes' D fragments
back as (RHS, spin, colour).  The result must equal the hop written the way
the FP32 lanes kernel computes it: the rank-2 projection (project2), the
colour multiply by U (forward) or U^dag (backward), and the reconstruction
(accum2), weighted by the FP16 record norms and the factor 2 of mu = 3.
"""

import numpy as np
import pytest


def project2(mu, C, s):
    """rows 0, 1 of (1 + C g_mu) psi (mu = 3 without its factor 2); s[spin][colour]."""
    if mu == 0:
        return np.array([s[0] + C * s[3], s[1] + C * s[2]])
    if mu == 1:
        return np.array([s[0] - 1j * C * s[3], s[1] + 1j * C * s[2]])
    if mu == 2:
        return np.array([s[0] - 1j * C * s[2], s[1] - 1j * C * s[3]])
    return np.array([s[0], s[1]]) if C > 0 else np.array([s[2], s[3]])


def accum2(mu, C, acc, uh, w):
    u0, u1 = uh
    if mu == 3:
        if C > 0:
            acc[0] += w * u0
            acc[1] += w * u1
        else:
            acc[2] += w * u0
            acc[3] += w * u1
        return
    acc[0] += w * u0
    acc[1] += w * u1
    if mu == 0:
        acc[2] += C * w * u1
        acc[3] += C * w * u0
    elif mu == 1:
        acc[2] += -1j * C * w * u1
        acc[3] += 1j * C * w * u0
    else:
        acc[2] += 1j * C * w * u0
        acc[3] += 1j * C * w * u1


def mma_rows(mu, C, v, w):
    """the kernel's A words for output spins 0..3 (complex numbers); v = spins 0..3 of one colour."""
    s0, s1, s2, s3 = v
    if mu == 0:
        h0, h1 = s0 + C * s3, s1 + C * s2
    elif mu == 1:
        h0, h1 = s0 - 1j * C * s3, s1 + 1j * C * s2
    elif mu == 2:
        h0, h1 = s0 - 1j * C * s2, s1 - 1j * C * s3
    else:
        h0, h1 = (s0, s1) if C > 0 else (s2, s3)
    h0, h1 = w * h0, w * h1
    if mu == 3:
        return [h0, h1, 0, 0] if C > 0 else [0, 0, h0, h1]
    if mu == 0:
        return [h0, h1, C * h1, C * h0]
    if mu == 1:
        return [h0, h1, -1j * C * h1, 1j * C * h0]
    return [h0, h1, 1j * C * h0, 1j * C * h1]


def byte_perm_halves(x, y, sel):
    """__byte_perm on words given as (lo, hi) half pairs: 0x5410 -> (x.lo, y.lo), 0x3276 -> (y.hi, x.hi)."""
    if sel == 0x5410:
        return (x[0], y[0])
    assert sel == 0x3276
    return (y[1], x[1])


@pytest.mark.parametrize("dag", [False, True])
@pytest.mark.parametrize("nact", [8, 5])
def test_lane_fragments_reproduce_the_hop(dag, nact):
    rng = np.random.default_rng(7 + dag + nact)
    CF = 1 if dag else -1
    psi = rng.normal(size=(8, 8, 4, 3)) + 1j * rng.normal(size=(8, 8, 4, 3))  # [hop][rhs][spin][colour]
    norm = rng.uniform(0.1, 3.0, size=(8, 8))
    norm[:, 3] *= 1e-3  # a RHS whose neighbours differ widely in scale
    norm[2, 4] *= 1e-5
    U = rng.normal(size=(8, 3, 3)) + 1j * rng.normal(size=(8, 3, 3))  # link of hop q (backward: U(x - mu))
    act = np.arange(8) < nact

    # reference: the lanes kernel's formulas
    ref = np.zeros((8, 4, 3), dtype=complex)
    for r in range(8):
        if not act[r]:
            continue
        for q in range(8):
            mu, back = q // 2, q % 2
            C = -CF if back else CF
            h = project2(mu, C, psi[q, r])
            Uop = U[q].conj().T if back else U[q]
            uh = np.array([Uop @ h[0], Uop @ h[1]])
            accum2(mu, C, ref[r], uh, norm[q, r] * (2.0 if mu == 3 else 1.0))

    # staged link pairs: element k = (a, b) -> x = (re, re), y = (-sgn im, sgn im), sgn = -1 backward
    def staged(q, k):
        v = U[q][k // 3, k % 3]
        sgn = -1.0 if q % 2 else 1.0
        return (v.real, v.real), (-sgn * v.imag, sgn * v.imag)

    m = np.where(act, norm.max(axis=0), 0.0)  # per-RHS scale (max over the 8 hops)
    D = np.zeros((2, 32, 4))  # [tile][lane][c0..c3]
    for mu in range(4):
        Afull = np.zeros((2, 16, 16))
        Bfull = np.zeros((16, 8))
        for lane in range(32):
            g, t = lane >> 2, lane & 3
            r = g
            ca = g >> 1
            bval = ca < 3 and t < 3
            sel = 0x3276 if g & 1 else 0x5410
            kf, kb = (ca * 3 + t, t * 3 + ca) if bval else (0, 0)
            words = {}
            for back in (0, 1):
                q = 2 * mu + back
                C = -CF if back else CF
                on = act[r] and t < 3
                v = psi[q, r, :, t] if on else np.zeros(4)
                w = norm[q, r] / m[r] * (2.0 if mu == 3 else 1.0) if act[r] else 0.0
                words[back] = mma_rows(mu, C, v, w)
            bw = []
            for back, k in ((0, kf), (1, kb)):
                x, y = staged(2 * mu + back, k)
                bw.append(byte_perm_halves(x, y, sel) if bval else (0.0, 0.0))
            # a0 = (row g, cols 2t..), a1 = (row g + 8, cols 2t..), a2 = (row g, cols 2t + 8..), a3 = (row g + 8, ..)
            for j in range(2):
                for row, col, z in ((g, 2 * t, words[0][2 * j]), (g + 8, 2 * t, words[0][2 * j + 1]),
                                    (g, 2 * t + 8, words[1][2 * j]), (g + 8, 2 * t + 8, words[1][2 * j + 1])):
                    z = complex(z)
                    Afull[j, row, col] = z.real
                    Afull[j, row, col + 1] = z.imag
            for back in (0, 1):
                lo, hi = bw[back]
                Bfull[2 * t + 8 * back, g] = lo
                Bfull[2 * t + 8 * back + 1, g] = hi
        for j in range(2):
            Dt = Afull[j] @ Bfull
            for lane in range(32):
                g, t = lane >> 2, lane & 3
                D[j, lane] += [Dt[g, 2 * t], Dt[g, 2 * t + 1], Dt[g + 8, 2 * t], Dt[g + 8, 2 * t + 1]]
    out = np.zeros((8, 4, 3), dtype=complex)
    for lane in range(32):
        g, t = lane >> 2, lane & 3
        if t == 3:
            assert np.all(D[:, lane] == 0)  # the pad column
            continue
        for j in range(2):
            out[g, 2 * j, t] = m[g] * complex(D[j, lane, 0], D[j, lane, 1])
            out[g, 2 * j + 1, t] = m[g] * complex(D[j, lane, 2], D[j, lane, 3])
    np.testing.assert_allclose(out, ref, rtol=0, atol=1e-12 * np.abs(ref).max())
    assert np.all(out[~act] == 0)


def test_smem_and_grid_bounds():
    """Shared memory per block and the partial-sum count the engine allocates."""
    link_slot, sites, hops = 72, 32, 8  # 4 warps x 8 sites
    smem = sites * hops * link_slot + sites * hops * 4 + sites * 4 + 4 * 8 * 8  # links, nb, ok, sred
    assert smem <= 48 * 1024  # static shared memory limit
    for vh in (4 * 6 * 4 * 8 // 2, 24 ** 3 * 48 // 2, 16 ** 3 * 32 // 2, 7):
        nblk = -(-vh // sites) * 2  # both parities
        assert nblk <= vh + 64
