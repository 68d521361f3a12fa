"""Host-side bounds checks of the warp-tile TMA hop (jaxqft_b200/csrc/wl_reftile.cuh), no GPU.

Each warp walks tiles of 16 consecutive sites of a t-row in four stages (the
tile itself, then the tiles at x -/+ e_mu for mu = 0, 1, 2), each staged by 2D
tensor-map copies (boxes of 24 lines of 128 bytes, 128-byte swizzle) into its
own double-buffered slots.  These tests restate the kernel's layout and index
arithmetic and check, for lattices with Lt a multiple of 16 and several RHS:

* the warps' tiles cover every (rhs, site) exactly once;
* every copy's line coordinate and box stay inside the field viewed as 128-byte
  lines, with x coordinate 0 (16-byte aligned), and the neighbour rows equal the
  rows of x -/+ e_mu with periodic wrap;
* the t-neighbours the kernel reads from global memory (t + 1 of the tile's last
  site, t - 1 of its first; with one tile per row these wrap into the tile
  itself and are still read from global memory) are inside the field;
* every swizzled read (site < 16, component < 12) lands inside its 3072-byte
  box, and the warps' slots plus barrier header and alignment slack fit the
  dynamic shared memory the launcher requests (and the 227 KB limit).
"""

import itertools

import numpy as np
import pytest

TILE, WARPS, BOX, BUFS, STAGES = 16, 4, 16 * 192, 2, 4
WARP_BYTES = BUFS * 2 * BOX
SMEM = 128 + 1024 + WARPS * WARP_BYTES


def swz_psi(site, comp):
    o = site * 192 + comp * 16
    line = o >> 7
    j = ((o >> 4) & 7) ^ (line & 7)
    return (line << 7) + (j << 4)


def tile_stage(L, tiles_per_rhs, wid, nw, k):
    tile = wid + (k // STAGES) * nw
    q = k % STAGES
    rhs = tile // tiles_per_rhs
    rem = tile - rhs * tiles_per_rhs
    tpr = L[3] // TILE
    row = rem // tpr
    return rhs, row, (rem - row * tpr) * TILE, q


def tile_line(L, V, rhs, row, t0):
    return ((rhs * V + row * L[3] + t0) * 3) >> 1


def stride_row(L):
    return [L[1] * L[2], L[2], 1]


def row_coords(L, row):
    return row // (L[1] * L[2]), (row // L[2]) % L[1], row % L[2]


SHAPES = [(2, 4, 2, 16), (4, 2, 6, 32), (2, 2, 4, 48), (3, 5, 7, 16), (24, 24, 24, 48), (16, 16, 16, 32)]


@pytest.mark.parametrize("L,nrhs", [(s, n) for s in SHAPES for n in (1, 2, 3)])
def test_tiles_cover_and_copies_stay_in_bounds(L, nrhs):
    V = int(np.prod(L))
    tiles_per_rhs = V // TILE
    ntiles = tiles_per_rhs * nrhs
    lines = nrhs * V * 3 // 2
    assert 24 * 128 == BOX and (TILE * 3) % 2 == 0
    big = V > 100000
    blocks = min((ntiles + WARPS - 1) // WARPS, 4 * 148)
    nw = blocks * WARPS
    covered = np.zeros(nrhs * V, dtype=np.int32) if not big else None
    wids = range(nw) if not big else [0, 1, nw // 2, nw - 1]
    for wid in wids:
        my = (ntiles - 1 - wid) // nw + 1 if wid < ntiles else 0
        for k in range(STAGES * my):
            rhs, row, t0, q = tile_stage(L, tiles_per_rhs, wid, nw, k)
            assert 0 <= rhs < nrhs and 0 <= row < V // L[3] and 0 <= t0 <= L[3] - TILE
            if q == 0:
                rows = [row]
                if covered is not None:
                    covered[rhs * V + row * L[3] + t0: rhs * V + row * L[3] + t0 + TILE] += 1
            else:
                mu = q - 1
                st, Lm = stride_row(L)[mu], L[mu]
                xm = (row // st) % Lm
                rp = row + (-(Lm - 1) * st if xm == Lm - 1 else st)
                rm = row + ((Lm - 1) * st if xm == 0 else -st)
                c = list(row_coords(L, row))
                cp, cm = c.copy(), c.copy()
                cp[mu] = (c[mu] + 1) % Lm
                cm[mu] = (c[mu] - 1) % Lm
                assert list(row_coords(L, rp)) == cp and list(row_coords(L, rm)) == cm
                rows = [rp, rm]
            for r in rows:
                y = tile_line(L, V, rhs, r, t0)
                assert 0 <= y and y + 24 <= lines < 2 ** 31
                assert ((rhs * V + r * L[3] + t0) * 3) % 2 == 0  # integral line start
            if q == 0:  # t-neighbours outside the tile
                for i, d in ((TILE - 1, +1), (0, -1)):
                    t = t0 + i
                    tn = (t + d) % L[3]
                    f = rhs * V + row * L[3] + tn
                    assert 0 <= f < nrhs * V
                    assert (tn < t0 or tn >= t0 + TILE) or L[3] == TILE
    if covered is not None:
        assert (covered == 1).all()


def test_swizzled_reads_and_shared_memory_fit():
    offs = [swz_psi(i, c) for i, c in itertools.product(range(TILE), range(12))]
    assert min(offs) >= 0 and max(offs) + 16 <= BOX
    assert len(set(offs)) == len(offs)  # a bijection of the box's 16-byte chunks it uses
    assert BOX % 1024 == 0 and (2 * BOX) % 1024 == 0  # every box starts on a swizzle atom
    # barriers (8 bytes per warp and buffer) fit the 128-byte header; slack <= 1023 bytes
    assert WARPS * BUFS * 8 <= 128
    assert 128 + 1023 + WARPS * WARP_BYTES <= SMEM <= 227 * 1024
