"""The warp-tile TMA kernel of the drop-in operators (ref_tile_kernel, selected
with WL_REF_HOP=tile, used when every site is targeted and Lt is a multiple of
16) against the numpy oracle: D, D^dag and the hopping term on lattices whose
t-rows hold one, two and three tiles, with several right-hand sides (tile rows
of different fields), periodic and complex boundary phases in every direction
(the tile-edge t-neighbours come from global memory, the rest from the staged
tiles), 1e-13 relative (jaxqft/fermions/wilson.py:171-284).  The kernel choice
is read once per process, so the checks run in a child process."""

import os
import subprocess
import sys

import numpy as np
import pytest

from oracle import wilson as W
from tests.conftest import ROOT, rel

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("CUDA device required", allow_module_level=True)

CASES = [
    ((2, 4, 2, 16), (1, 1, 1, -1), 3),
    ((4, 2, 6, 32), (1, 1j, 1, -1), 2),
    ((2, 2, 4, 48), (complex(np.cos(0.7), np.sin(0.7)), 1, -1, 1j), 1),
]


def check_all():
    """Runs in the child process (WL_REF_HOP=tile); raises on a mismatch."""
    from jaxqft_b200.lib import WilsonContext

    for shape, bc, nrhs in CASES:
        rng = np.random.default_rng(sum(shape))
        U = W.hot_links(rng, shape, 1, 0.3)
        psi = W.gaussian_spinor(rng, shape, nrhs)
        bc64 = tuple(complex(np.complex64(complex(b))) for b in bc)  # as the theory layer passes them
        mass = -0.2
        ctx = WilsonContext(shape, bc=bc64)
        gauge = ctx.gauge(torch.from_numpy(U[0]))
        x = torch.from_numpy(psi).cuda()
        D = ctx.apply("D", gauge, mass, x).cpu().numpy()
        Dd = ctx.apply("DDAG", gauge, mass, x).cpu().numpy()
        H = ctx.apply("HOP", gauge, mass, x).cpu().numpy()
        ctx.synchronize()  # raises if a bounded wait of the kernel ran out
        for r in range(nrhs):
            assert rel(D[r], W.apply_D(U, psi[r:r + 1], mass, bc64)[0]) < 1e-13, (shape, r, "D")
            assert rel(Dd[r], W.apply_Ddag(U, psi[r:r + 1], mass, bc64)[0]) < 1e-13, (shape, r, "Ddag")
            assert rel(H[r], W.apply_hop(U, psi[r:r + 1], bc64)[0]) < 1e-13, (shape, r, "hop")
    print("tile kernel ok")


def test_tile_kernel_operators():
    env = dict(os.environ, WL_REF_HOP="tile")
    res = subprocess.run([sys.executable, "-c", "import tests.test_gpu_tile_hop as T; T.check_all()"], cwd=ROOT,
                         env=env, capture_output=True, text=True, timeout=600)
    assert res.returncode == 0 and "tile kernel ok" in res.stdout, res.stdout[-2000:] + res.stderr[-4000:]
