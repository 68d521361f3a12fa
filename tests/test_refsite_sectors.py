"""Host-side restatement of the sector loads of the drop-in pair kernel (ld_pair_spins in
jaxqft_b200/csrc/wl_refsite.cuh), no GPU.

A site of the caller's complex128 [4][3] spinor is 192 bytes = six 32-byte sectors; sector k
holds reals [4k, 4k + 4), i.e. complex values z[2k], z[2k + 1] with z[3 spin + colour].  Each
load instruction of the pair reads one 64-byte piece (thread j one sector of it); the pair then
swaps values with one xor-shuffle per double.  This test replays the two threads' loads,
shuffles and selections for every hop type and checks that thread j ends with the spins the
pair decomposition needs (pair_spin1 / pair_spin2): a = spin j (or 2 + j for mu = 3, C < 0),
b = spin 3 - j (mu = 0, 1) or 2 + j (mu = 2).  It also checks that every piece is one aligned
64-byte block, so an instruction touches a single 128-byte line per site.
"""

import pytest


def sectors_loaded(mu, C, j):
    """(r0, r1, r2) sector indices thread j loads (None: not loaded)."""
    if mu < 3:
        return j, 3 - j, (5 - j if mu < 2 else 4 + j)
    if C > 0:
        return j, 3 - j, None
    return None, 3 - j, 4 + j


def reals(z, sec):
    """the four doubles of sector sec: re/im of z[2 sec], z[2 sec + 1]."""
    if sec is None:
        return [None] * 4
    a, b = z[2 * sec], z[2 * sec + 1]
    return [a.real, a.imag, b.real, b.imag]


def pick(j, x0, x1):
    return x1 if j else x0


def replay(mu, C, z):
    regs = {}
    for j in (0, 1):
        s0, s1, s2 = sectors_loaded(mu, C, j)
        regs[j] = (reals(z, s0), reals(z, s1), reals(z, s2))
    out = {}
    for j in (0, 1):
        r0, r1, r2 = regs[j]
        o0, o1, o2 = regs[1 - j]  # the partner's registers (what the shuffle reads)
        if mu < 2:
            # snd = j ? (k < 2 ? r0[k] : r2[k]) : r1[k]
            x = [((o0[k] if k < 2 else o2[k]) if (1 - j) else o1[k]) for k in range(4)]
            a = [pick(j, r0[0], r0[2]), pick(j, r0[1], r0[3]), pick(j, r0[2], r1[0]), pick(j, r0[3], r1[1]),
                 pick(j, x[0], r1[2]), pick(j, x[1], r1[3])]
            b = [pick(j, x[2], x[0]), pick(j, x[3], x[1]), pick(j, r2[0], x[2]), pick(j, r2[1], x[3]),
                 pick(j, r2[2], r2[0]), pick(j, r2[3], r2[1])]
        elif mu == 2:
            x = [(o0[k] if (1 - j) else o2[2 + k]) for k in range(2)]
            a = [pick(j, r0[0], r0[2]), pick(j, r0[1], r0[3]), pick(j, r0[2], r1[0]), pick(j, r0[3], r1[1]),
                 pick(j, x[0], r1[2]), pick(j, x[1], r1[3])]
            b = [pick(j, r1[0], x[0]), pick(j, r1[1], x[1]), pick(j, r1[2], r2[0]), pick(j, r1[3], r2[1]),
                 pick(j, r2[0], r2[2]), pick(j, r2[1], r2[3])]
        elif C > 0:
            x = [o0[k] for k in range(2)]
            a = [pick(j, r0[0], r0[2]), pick(j, r0[1], r0[3]), pick(j, r0[2], r1[0]), pick(j, r0[3], r1[1]),
                 pick(j, x[0], r1[2]), pick(j, x[1], r1[3])]
            b = None
        else:
            x = [o2[2 + k] for k in range(2)]
            a = [pick(j, r1[0], x[0]), pick(j, r1[1], x[1]), pick(j, r1[2], r2[0]), pick(j, r1[3], r2[1]),
                 pick(j, r2[0], r2[2]), pick(j, r2[1], r2[3])]
            b = None
        out[j] = (a, b)
    return out


def spin_reals(z, s):
    return [v for c in range(3) for v in (z[3 * s + c].real, z[3 * s + c].imag)]


@pytest.mark.parametrize("mu,C", [(0, 1), (0, -1), (1, 1), (1, -1), (2, 1), (2, -1), (3, 1), (3, -1)])
def test_pair_ends_with_its_spins(mu, C):
    z = [complex(2 * i + 1, 2 * i + 2) for i in range(12)]  # distinct values
    out = replay(mu, C, z)
    for j in (0, 1):
        a, b = out[j]
        s1 = (2 + j) if (mu == 3 and C < 0) else j  # pair_spin1
        assert a == spin_reals(z, s1), (mu, C, j)
        if mu < 3:
            s2 = 2 + j if mu == 2 else 3 - j  # pair_spin2
            assert b == spin_reals(z, s2), (mu, C, j)


@pytest.mark.parametrize("mu,C", [(0, 1), (1, -1), (2, 1), (3, 1), (3, -1)])
def test_pieces_are_aligned_64_byte_blocks(mu, C):
    s = [sectors_loaded(mu, C, j) for j in (0, 1)]
    for k in range(3):
        pair = {s[0][k], s[1][k]} - {None}
        if not pair:
            continue
        assert min(pair) % 2 == 0 and max(pair) - min(pair) <= 1  # one 64-byte block
        for site in range(4):  # site base 192 s: the block stays in one 128-byte line
            lo = 192 * site + 32 * min(pair)
            assert lo // 128 == (lo + 63) // 128


def test_store_sectors():
    """pair_store_sect: thread j holds sectors 3j..3j+2 (o[0..11]); sector 1 of thread 0 and
    sector 4 of thread 1 (both o[4..7]) are swapped; thread j then writes v = sectors j, 2+j, 4+j
    to doubles 8 p + 4 j, p = 0, 1, 2."""
    site = [float(k) for k in range(24)]  # the values each double of the site should end with
    o = {j: site[12 * j:12 * j + 12] for j in (0, 1)}
    ex = {j: o[j][:4] + o[1 - j][4:8] + o[j][8:] for j in (0, 1)}  # after the shuffle of o[4..7]
    out = [None] * 24
    for j in (0, 1):
        oo = ex[j]
        v = [None] * 12
        for k in range(4):
            v[k] = pick(j, oo[k], oo[4 + k])
            v[4 + k] = pick(j, oo[8 + k], oo[k])
            v[8 + k] = pick(j, oo[4 + k], oo[8 + k])
        for p in range(3):
            for k in range(4):
                out[8 * p + 4 * j + k] = v[4 * p + k]
    assert out == site
