"""Host-side bounds checks of the row-staged FP64 hop (jaxqft_b200/csrc/wl_rowhop.cuh), no GPU.

The kernel stages, per (x, y, z) row of Lt sites and per direction, spinor rows
by 2D tensor-map copies with the 128-byte swizzle and link rows by 1D bulk
copies into shared-memory stage buffers.  These tests restate its layout
arithmetic and check, for every even Lt the host accepts (2 <= Lt <= kRowMaxLt):

* every swizzled spinor read (site < Lt, component < 12) lands inside the bytes
  the tensor-map box writes (1.5 Lt lines of 128 bytes) and inside its padded
  slot; the swizzle is a bijection of the row's 16-byte chunks;
* the link rows (144 Lt bytes each, forward and backward) fit after the two
  spinor slots inside one stage, and kRowBufs stages plus the barrier header
  and the 1024-byte alignment slack fit in the 227 KB a block may use;
* the box is legal for TMA: inner extent 16 FP64 = 128 bytes (the swizzle span),
  at most 256 rows, x coordinate 0 (16-byte aligned), and a bulk copy's size and
  its shared-memory destination offsets are multiples of 16 bytes;
* the neighbour-row arithmetic with periodic wrap stays inside [0, rows) and
  equals the rows of x +- e_mu, and the row coordinate of every copy stays
  inside the field viewed as 128-byte lines.
"""

import numpy as np
import pytest

K_ROW_BUFS = 2  # WL_ROW_BUFS
K_ROW_MAX_LT = min((220 * 1024) // (672 * K_ROW_BUFS), 148)
SMEM_LIMIT = 227 * 1024


def row_psi_pad(lt):
    return ((192 * lt + 1023) // 1024) * 1024


def row_stage_bytes(lt):
    return ((2 * row_psi_pad(lt) + 288 * lt + 1023) // 1024) * 1024


def swz_psi(site, comp):
    """Byte offset of (site, component) in a swizzled row (swz_psi)."""
    o = site * 192 + comp * 16
    line = o >> 7
    j = ((o >> 4) & 7) ^ (line & 7)
    return (line << 7) + (j << 4)


@pytest.mark.parametrize("lt", list(range(2, K_ROW_MAX_LT + 1, 2)))
def test_stage_layout_in_bounds(lt):
    spad = row_psi_pad(lt)
    box_lines = lt * 3 // 2
    assert box_lines <= 256 and box_lines * 128 == 192 * lt  # TMA box rows; whole lines for even Lt
    offs = np.array([swz_psi(s, c) for s in range(lt) for c in range(12)])
    assert offs.min() >= 0 and offs.max() + 16 <= box_lines * 128 <= spad
    assert np.unique(offs).size == offs.size  # the swizzle permutes the row's chunks
    lk = 144 * lt
    stage = row_stage_bytes(lt)
    assert 2 * spad + 2 * lk <= stage and stage % 1024 == 0
    assert (2 * spad) % 16 == 0 and (2 * spad + lk) % 16 == 0 and lk % 16 == 0  # bulk copy dst / size
    assert (144 * lt) % 16 == 0 and 144 % 16 == 0  # link rows start at (mu V + row Lt) * 144 bytes: 16-aligned src
    smem = 128 + 1024 + K_ROW_BUFS * stage  # barrier header, alignment slack, stage buffers
    assert smem <= SMEM_LIMIT, (lt, smem)
    assert 3 * lt <= 3 * K_ROW_MAX_LT <= 1024  # threads per block within the launch bounds


@pytest.mark.parametrize("L", [(2, 2, 2, 4), (4, 4, 4, 8), (2, 4, 6, 4), (6, 2, 4, 10), (24, 24, 24, 48)],
                         ids=lambda s: "x".join(map(str, s)))
def test_neighbour_rows_and_copy_coordinates(L):
    Lx, Ly, Lz, Lt = L
    nrows = Lx * Ly * Lz
    stride_row = (Ly * Lz, Lz, 1)
    rows = np.arange(nrows)
    x = np.array(np.unravel_index(rows, (Lx, Ly, Lz)))
    for mu in range(3):
        lm, stride = L[mu], stride_row[mu]
        xm = (rows // stride) % lm
        rp = rows + np.where(xm == lm - 1, -(lm - 1) * stride, stride)
        rm = rows + np.where(xm == 0, (lm - 1) * stride, -stride)
        for r, d in ((rp, +1), (rm, -1)):
            assert r.min() >= 0 and r.max() < nrows
            y = x.copy()
            y[mu] = (y[mu] + d) % lm
            assert np.array_equal(r, np.ravel_multi_index(y, (Lx, Ly, Lz))), (L, mu, d)
    # tensor-map rows: line0 + row * lpr with a box of lpr lines stays inside the field's lines
    for nrhs in (1, 3):
        lines = nrhs * Lx * Ly * Lz * Lt * 3 // 2
        lpr = Lt * 3 // 2
        line0 = np.arange(nrhs)[:, None] * (Lx * Ly * Lz * Lt) * 3 // 2
        last = line0 + rows[None, :] * lpr + lpr
        assert last.max() <= lines and lines < 2 ** 31
