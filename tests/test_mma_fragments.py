"""Host-side restatement of the tensor-core FP16 hop (jaxqft_b200/csrc/wl_hop_mma.cuh), no GPU.

The kernel computes one site's hop over 16 RHS as 16 mma.sync m16n8k16 tiles:
for each mu, four output-spin tiles whose rows are the 16 RHS and whose K holds
the forward and backward hop's projected colour components; lane (g, t) holds
colour t of RHS g and g + 8.  This test rebuilds, in float64, every lane's A
words (``mma_project``: weighted rank-2 projection), B words (``bword`` of the
staged link element, its dagger for the backward hop, and the lower spins'
coefficient ``cmul_unit<LowerKappa>``), the per-tile matrices of the PTX
fragment layout of m16n8k16 (A: rows g / g + 8, columns 2t, 2t + 1 and 2t + 8,
2t + 9; B: rows 2t, 2t + 1 and 2t + 8, 2t + 9, column g; D: rows g / g + 8,
columns 2t, 2t + 1), multiplies them, and reads the lanes' D fragments back as
(RHS, spin, colour).  The result must equal the hop written the way the FP32
lanes kernel computes it: the rank-2 projection (project2), the colour
multiply by U (forward) or U^dag (backward), and the reconstruction (accum2),
weighted by the FP16 record norms and the factor 2 of mu = 3.  The shared
memory layout (record slots with the r ^ 2t swizzle) and the cp.async
assignment are checked too.
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


def proj_rows(mu, C, v, w):
    """the kernel's A words of one record chunk: w * rows 0, 1 of (1 + C g_mu) psi (``mma_project``)."""
    h0, h1 = project2(mu, C, v)
    return w * h0, w * h1


KAPPA = {0: 1, 1: -1, 2: 1j, 3: -1j}  # cmul_unit<K>


def lower_kappa(mu, C):
    """``LowerKappa``: coefficient of the lower spins, mu = 0: C, mu = 1: -iC, mu = 2: iC."""
    if mu == 0:
        return 0 if C > 0 else 1
    if mu == 1:
        return 3 if C > 0 else 2
    return 2 if C > 0 else 3


def bword(e, imc):
    """B word of a lane for complex element e: column (a, re) -> (re, -im), column (a, im) -> (im, re)."""
    return (e.imag, e.real) if imc else (e.real, -e.imag)


def swizzle_ok():
    """chunk (q, t, r) stored at RHS index r ^ 2t: a permutation, and the 16-byte reads of each
    quarter-warp (8 lanes: g in {2p, 2p+1}, t in 0..2) hit distinct 16-byte bank groups."""
    for t in range(3):
        assert sorted(r ^ (2 * t) for r in range(16)) == list(range(16))
    for p in range(4):
        for hi in (0, 8):
            groups = [((g + hi) ^ (2 * t)) % 8 for g in (2 * p, 2 * p + 1) for t in range(3)]
            assert len(set(groups)) == len(groups)


def test_smem_swizzle_conflict_free():
    swizzle_ok()


@pytest.mark.parametrize("dag", [False, True])
@pytest.mark.parametrize("nact", [16, 11])
def test_lane_fragments_reproduce_the_hop(dag, nact):
    rng = np.random.default_rng(7 + dag + nact)
    CF = 1 if dag else -1
    NR = 16
    psi = rng.normal(size=(8, NR, 4, 3)) + 1j * rng.normal(size=(8, NR, 4, 3))  # [hop][rhs][spin][colour]
    norm = rng.uniform(0.1, 3.0, size=(8, NR))
    norm[:, 3] *= 1e-3  # a RHS whose neighbours differ widely in scale
    norm[2, 4] *= 1e-5
    norm[5, 12] *= 1e-4
    U = rng.normal(size=(8, 3, 3)) + 1j * rng.normal(size=(8, 3, 3))  # staged link of hop q (backward: U(x - mu))
    act = np.arange(NR) < nact

    # reference: the lanes kernel's formulas
    ref = np.zeros((NR, 4, 3), dtype=complex)
    for r in range(NR):
        if not act[r]:
            continue
        for q in range(8):
            mu, back = q // 2, q % 2
            C = -CF if back else CF
            h = project2(mu, C, psi[q, r])
            Uop = U[q].conj().T if back else U[q]
            uh = np.array([Uop @ h[0], Uop @ h[1]])
            accum2(mu, C, ref[r], uh, norm[q, r] * (2.0 if mu == 3 else 1.0))

    nrm = np.where(act[None, :], norm, 0.0)  # zero-filled norms of inactive RHS
    m = nrm.max(axis=0)
    inv = np.where(m > 0, 1.0 / np.where(m > 0, m, 1.0), 0.0)
    D = np.zeros((4, 32, 4))  # [spin tile][lane][d0..d3]
    for mu in range(4):
        qf, qb = 2 * mu, 2 * mu + 1
        A = np.zeros((2, 16, 16))  # row tiles 0, 1
        B = {k: np.zeros((16, 8)) for k in ("up", "lo", "lo_neg")}
        for lane in range(32):
            g, t = lane >> 2, lane & 3
            # A words (rows g, g + 8; forward cols 2t.., backward cols 2t + 8..)
            if t < 3:
                for row, r in ((g, g), (g + 8, g + 8)):
                    for q, col0 in ((qf, 0), (qb, 8)):
                        C = CF if q == qf else -CF
                        v = psi[q, r, :, t] if act[r] else np.zeros(4)
                        w = nrm[q, r] * inv[r] * (2.0 if mu == 3 else 1.0)
                        h0, h1 = proj_rows(mu, C, v, w)
                        for j, h in ((0, h0), (1, h1)):
                            A[j, row, col0 + 2 * t] = h.real
                            A[j, row, col0 + 2 * t + 1] = h.imag
            # B words: column g, rows 2t, 2t + 1 (forward) and 2t + 8, 2t + 9 (backward)
            a, imc = g >> 1, g & 1
            uf = U[qf][a, t] if (a < 3 and t < 3) else 0.0
            vb = np.conj(U[qb][t, a]) if (a < 3 and t < 3) else 0.0
            if mu < 3:
                K = lower_kappa(mu, CF)
                words = {"up": (uf, vb), "lo": (KAPPA[K] * uf, KAPPA[K ^ 1] * vb)}
            else:
                words = {"up": (uf if CF > 0 else 0.0, vb if CF < 0 else 0.0),
                         "lo": (uf if CF < 0 else 0.0, vb if CF > 0 else 0.0)}
            words["lo_neg"] = (-words["lo"][0], -words["lo"][1])
            for k, (ef, eb) in words.items():
                for e, row0 in ((ef, 2 * t), (eb, 2 * t + 8)):
                    lo, hi = bword(complex(e), imc)
                    B[k][row0, g] = lo
                    B[k][row0 + 1, g] = hi
        tiles = {0: (0, "up"), 1: (1, "up")}
        if mu == 0:
            tiles.update({2: (1, "lo"), 3: (0, "lo")})
        elif mu == 1:
            tiles.update({2: (1, "lo"), 3: (0, "lo_neg")})
        else:
            tiles.update({2: (0, "lo"), 3: (1, "lo")})
        for s, (j, k) in tiles.items():
            Dt = A[j] @ B[k]
            for lane in range(32):
                g, t = lane >> 2, lane & 3
                D[s, lane] += [Dt[g, 2 * t], Dt[g, 2 * t + 1], Dt[g + 8, 2 * t], Dt[g + 8, 2 * t + 1]]
    out = np.zeros((NR, 4, 3), dtype=complex)
    for lane in range(32):
        g, t = lane >> 2, lane & 3
        if t == 3:
            assert np.all(D[:, lane] == 0)  # the pad column
            continue
        for s in range(4):
            out[g, s, t] = m[g] * complex(D[s, lane, 0], D[s, lane, 1])
            out[g + 8, s, t] = m[g + 8] * complex(D[s, lane, 2], D[s, lane, 3])
    np.testing.assert_allclose(out, ref, rtol=0, atol=1e-12 * np.abs(ref).max())
    assert np.all(out[~act] == 0)


def test_smem_and_grid_bounds():
    """Dynamic shared memory per block (MmaSmem) and the partial-sum count the engine allocates."""
    slot = 8 * 3 * 16 * 16 + 8 * 16 * 4  # chunks, norms
    warp = 2 * slot + 8 * 8 * 9 * 4 + 8 * 8 * 4 + 8 * 4  # two slots, links, nb, ok
    smem = 4 * warp + 4 * 16 * 8  # + sred
    assert smem % 16 == 0 and warp % 16 == 0
    assert 3 * smem <= 228 * 1024  # three resident blocks per SM
    for vh in (4 * 6 * 4 * 8 // 2, 24 ** 3 * 48 // 2, 16 ** 3 * 32 // 2, 7):
        nblk = -(-vh // 32) * 2  # 32 sites per block, both parities
        assert nblk <= vh + 64


def test_fetch_covers_every_chunk_once():
    """mma_fetch: lane L copies RHS L % 16 of hops 4 (L // 16) .. + 3, every colour, and their norms."""
    seen, norms = set(), set()
    for lane in range(32):
        r, h = lane & 15, lane >> 4
        for k in range(4):
            q = 4 * h + k
            for t in range(3):
                seen.add((q, t, r ^ (2 * t)))
            norms.add((r, q))  # S.norm[r][q]: a lane reads its RHS's eight norms as two 16-byte words
    assert len(seen) == 8 * 3 * 16 and len(norms) == 8 * 16
