"""Host-side checks of the kernels' index arithmetic (no GPU).

The device code decodes compact site indices with multiply-shift division
(make_fastdiv / fdiv in jaxqft_b200/csrc/wl_common.cuh), gathers neighbours by
index arithmetic (neighbor) and sweeps the FP64 update hop in a tiled order
(tiled_compact).  These tests restate those formulas exactly, with the same
32-bit multiplier and shift, and check them:

* fdiv(n, d) == n // d for every divisor 1..4096, at every multiple boundary
  near the top of the index range and on a dense set of small n;
* site_from_compact and neighbor reproduce the reference's even/odd index lists
  and compact neighbour maps (su3_wilson_nf2.py:831-882, restated with numpy as
  the reference builds them) on many even lattice shapes;
* tiled_compact is a permutation of the compact sites, for the slab height Ty
  that wl_ctx_create picks (the largest divisor of Ly not above 8).
"""

import itertools

import numpy as np
import pytest

N_MAX = 1 << 31  # fdiv is exact for 0 <= n < 2^31; site indices stay below 2^30


def make_fastdiv(d):
    """(mul, shr) as in make_fastdiv: l = ceil(log2 d), mul = ceil(2^(31+l)/d)."""
    if d <= 1:
        return 0, 0
    l = 0
    while (1 << l) < d:
        l += 1
    return ((1 << (31 + l)) + d - 1) // d, l - 1


def fdiv(f, n):
    """__umulhi(n, mul) >> shr on uint64 arrays (n < 2^31, mul < 2^32)."""
    mul, shr = f
    n = np.asarray(n, dtype=np.uint64)
    if mul == 0:
        return n
    return ((n * np.uint64(mul)) >> np.uint64(32)) >> np.uint64(shr)


def test_fastdiv_matches_integer_division():
    small = np.arange(0, 1 << 16, dtype=np.uint64)
    for d in range(1, 4097):
        f = make_fastdiv(d)
        assert f[0] < (1 << 32)
        assert np.array_equal(fdiv(f, small), small // np.uint64(d)), d
        # the multiple boundaries k*d - 1, k*d of the top 2^16 quotients (the error term grows with n)
        kmax = (N_MAX - 1) // d
        k = np.arange(max(1, kmax - (1 << 16)), kmax + 1, dtype=np.uint64)
        for n in (k * np.uint64(d) - np.uint64(1), k * np.uint64(d)):
            n = n[n < np.uint64(N_MAX)]
            assert np.array_equal(fdiv(f, n), n // np.uint64(d)), d
        top = np.array([N_MAX - 1], dtype=np.uint64)
        assert fdiv(f, top)[0] == (N_MAX - 1) // d


class Geom:
    """The host-side geometry of wl_ctx_create."""

    def __init__(self, L):
        self.L = tuple(int(v) for v in L)
        self.V = int(np.prod(L))
        self.Vh = self.V // 2
        self.Lth = self.L[3] // 2
        self.strideRow = (self.L[1] * self.L[2], self.L[2], 1)
        self.Ty = next(d for d in range(8, 0, -1) if self.L[1] % d == 0)
        self.fd_lth, self.fd_l2, self.fd_l1 = (make_fastdiv(self.Lth), make_fastdiv(self.L[2]),
                                               make_fastdiv(self.L[1]))
        self.fd_ty, self.fd_l0 = make_fastdiv(self.Ty), make_fastdiv(self.L[0])


def site_from_compact(g, parity, c):
    """Vectorised restatement of site_from_compact: (row, x0, x1, x2, x3)."""
    c = np.asarray(c, dtype=np.int64)
    row = fdiv(g.fd_lth, c).astype(np.int64)
    th = c - row * g.Lth
    r2 = fdiv(g.fd_l2, row).astype(np.int64)
    x2 = row - r2 * g.L[2]
    x0 = fdiv(g.fd_l1, r2).astype(np.int64)
    x1 = r2 - x0 * g.L[1]
    x3 = 2 * th + ((parity + x0 + x1 + x2) & 1)
    return row, (x0, x1, x2, x3)


def neighbor(g, row, x, mu, d):
    """Restatement of neighbor: compact index of x + d e_mu in the other parity."""
    if mu == 3:
        t = x[3] + d
        t = np.where(t < 0, t + g.L[3], np.where(t >= g.L[3], t - g.L[3], t))
        return row * g.Lth + (t >> 1)
    xm = x[mu] + d
    r = row + d * g.strideRow[mu]
    r = np.where(xm < 0, r + g.L[mu] * g.strideRow[mu], np.where(xm >= g.L[mu], r - g.L[mu] * g.strideRow[mu], r))
    return r * g.Lth + (x[3] >> 1)


def tiled_compact(g, cl):
    cl = np.asarray(cl, dtype=np.int64)
    row_l = fdiv(g.fd_lth, cl).astype(np.int64)
    th = cl - row_l * g.Lth
    r1 = fdiv(g.fd_l2, row_l).astype(np.int64)
    z = row_l - r1 * g.L[2]
    r2 = fdiv(g.fd_ty, r1).astype(np.int64)
    yi = r1 - r2 * g.Ty
    yb = fdiv(g.fd_l0, r2).astype(np.int64)
    x = r2 - yb * g.L[0]
    row = (x * g.L[1] + yb * g.Ty + yi) * g.L[2] + z
    return row * g.Lth + th


def reference_maps(L):
    """The reference's even/odd flat index lists and compact neighbour maps
    (_build_checkerboard_indices and _build_checkerboard_neighbor_maps)."""
    parity = np.zeros(L, dtype=np.int64)
    for ax, n in enumerate(L):
        shp = [1] * 4
        shp[ax] = n
        parity = parity + np.arange(n).reshape(shp)
    flat = parity.reshape(-1)
    idx = [np.flatnonzero(flat % 2 == p) for p in (0, 1)]
    inv = [np.full(int(np.prod(L)), -1, dtype=np.int64) for _ in range(2)]
    for p in (0, 1):
        inv[p][idx[p]] = np.arange(idx[p].size)

    def shift(fi, mu, step):
        co = np.array(np.unravel_index(fi, L))
        co[mu] = (co[mu] + step) % L[mu]
        return np.ravel_multi_index(co, L)

    # maps[p][(mu, d)] = compact index, in parity 1-p, of the neighbour of each parity-p site
    maps = [{(mu, d): inv[1 - p][shift(idx[p], mu, d)] for mu in range(4) for d in (+1, -1)} for p in (0, 1)]
    return idx, maps


EXTENTS = (2, 4, 6, 8, 10, 12)
SHAPES = sorted(set(itertools.islice(
    (s for s in itertools.product(EXTENTS, repeat=4) if int(np.prod(s)) <= 6000), 0, None)))[::37] + [
    (4, 4, 4, 4), (2, 4, 6, 4), (8, 12, 6, 16), (4, 6, 10, 8), (16, 16, 16, 32)]


@pytest.mark.parametrize("L", SHAPES, ids=lambda s: "x".join(map(str, s)))
def test_decode_and_neighbours_match_reference_maps(L):
    g = Geom(L)
    idx, maps = reference_maps(L)
    c = np.arange(g.Vh)
    for p in (0, 1):
        row, x = site_from_compact(g, p, c)
        assert np.array_equal(np.ravel_multi_index(x, L), idx[p]), (L, p)  # compact order = ascending flat order
        for mu in range(4):
            for d in (+1, -1):
                nb = neighbor(g, row, x, mu, d)
                assert nb.min() >= 0 and nb.max() < g.Vh
                assert np.array_equal(nb, maps[p][(mu, d)]), (L, p, mu, d)


@pytest.mark.parametrize("L", SHAPES + [(24, 24, 24, 48), (12, 18, 6, 8), (6, 14, 4, 2)],
                         ids=lambda s: "x".join(map(str, s)))
def test_tiled_sweep_is_a_permutation(L):
    g = Geom(L)
    assert L[1] % g.Ty == 0 and 1 <= g.Ty <= 8
    t = tiled_compact(g, np.arange(g.Vh))
    assert t.min() >= 0 and t.max() < g.Vh
    assert np.array_equal(np.sort(t), np.arange(g.Vh)), L
