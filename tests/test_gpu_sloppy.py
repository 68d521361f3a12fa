"""The FP16 and FP32 iterated operators of the solver engine against the FP64
oracle, on Gaussian and on point-source fields (the latter have most sites
exactly zero, the hard case for per-site FP16 norms).

Tolerances (relative, Frobenius): FP64 1e-13; FP32 storage + 12-real links
1e-6 for D and D^dag applied to a spinor (the FP32 bound the port is held
to) and 2e-6 for the composite operators K, M, M^dag M and D^dag D, whose
cancellations (M = 1 - K K / m0^2 near the critical kappa) amplify the FP32
rounding of the intermediate field; FP16 storage (per-site norm) + 12-real
FP16 links with FP32 arithmetic 4e-3 per application of M^dag M.
"""

import numpy as np
import pytest

from oracle import wilson as W
from tests.conftest import load_golden, rel

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("CUDA device required", allow_module_level=True)

from jaxqft_b200.lib import Engine, WilsonContext  # noqa: E402

TOLS = {"double": 1e-13, "single": 2e-6, "half": 4e-3}
TOLS_D = {"double": 1e-13, "single": 1e-6, "half": 4e-3}  # D and D^dag applied to a spinor


def _fields(shape, seed):
    rng = np.random.default_rng(seed)
    gauss = W.gaussian_spinor(rng, shape, 1)[0]
    point = np.zeros_like(gauss)
    point[0, 0, 0, 0, 1, 2] = 1.0
    return {"gauss": gauss, "point": point}


@pytest.fixture(scope="module")
def setup():
    shape = (4, 4, 4, 8)
    rng = np.random.default_rng(7)
    U = W.hot_links(rng, shape, 1, 0.2)
    bc = (1, 1, 1, -1)
    ctx = WilsonContext(shape, bc=bc)
    gauge = ctx.gauge(torch.from_numpy(U[0]))
    return shape, U, bc, ctx, gauge


@pytest.mark.parametrize("inner", ["double", "single", "half"])
@pytest.mark.parametrize("src", ["gauss", "point"])
def test_eo_sloppy_operators(setup, inner, src):
    shape, U, bc, ctx, gauge = setup
    m = -0.2962963
    eng = Engine(ctx, gauge, 1, op="eo_normal", inner=inner)
    xe = W.project(_fields(shape, 1)[src][None], 0)
    refs = {
        0: W.K_block(U, xe, bc, 0),
        1: W.schur_even(U, xe, m, bc, normalized=True),
    }
    refs[2] = W.schur_even(U, refs[1], m, bc, normalized=True, dag=True)
    for stage, ref in refs.items():
        out = eng.debug_apply(stage, m, torch.from_numpy(xe[0])).cpu().numpy()
        assert rel(out, ref[0]) < TOLS[inner], (inner, src, stage, rel(out, ref[0]))
    eng.close()


@pytest.mark.parametrize("inner", ["double", "single", "half"])
def test_full_sloppy_operators(setup, inner):
    shape, U, bc, ctx, gauge = setup
    m = 0.1
    eng = Engine(ctx, gauge, 1, op="normal", inner=inner)
    for src, x in _fields(shape, 2).items():
        out = eng.debug_apply(3, m, torch.from_numpy(x)).cpu().numpy()
        err = rel(out, W.apply_D(U, x[None], m, bc)[0])
        assert err < TOLS_D[inner], (inner, src, "D", err)
        out = eng.debug_apply(5, m, torch.from_numpy(x)).cpu().numpy()
        err = rel(out, W.apply_Ddag(U, x[None], m, bc)[0])
        assert err < TOLS_D[inner], (inner, src, "Ddag", err)
        out = eng.debug_apply(4, m, torch.from_numpy(x)).cpu().numpy()
        assert rel(out, W.apply_normal(U, x[None], m, bc)[0]) < TOLS[inner], (inner, src)
    eng.close()


@pytest.mark.parametrize("inner", ["single", "half"])
@pytest.mark.parametrize("op", ["eo_normal", "normal"])
def test_point_source_solves_converge(setup, inner, op):
    shape, U, bc, ctx, gauge = setup
    m = -0.2962963
    eta = np.zeros((12, *shape, 4, 3), dtype=np.complex128)
    for k in range(12):
        eta[k, 0, 0, 0, 0, k // 3, k % 3] = 1.0
    if op == "eo_normal":
        b = ctx.apply("SCHUR_E_DAG", gauge, m, torch.from_numpy(eta), normalized=True)
    else:
        b = ctx.apply("DDAG", gauge, m, torch.from_numpy(eta))
    x, st = ctx.solve(gauge, b, m, op=op, tol=1e-10, maxiter=3000, inner=inner)
    assert all(s["status"] == 2 for s in st), st
    bn, xn = b.cpu().numpy(), x.cpu().numpy()
    for r in range(12):
        if op == "eo_normal":
            s = W.schur_even(U, xn[r][None], m, bc, normalized=True)
            Ax = W.schur_even(U, s, m, bc, normalized=True, dag=True)[0]
        else:
            Ax = W.apply_normal(U, xn[r][None], m, bc)[0]
        assert np.linalg.norm(bn[r] - Ax) / np.linalg.norm(bn[r]) <= 1e-10


def test_point_source_long_lattice_half():
    """Regression: on a long lattice a point-source Krylov vector decays below
    FLT_MIN far from the source; the FP16 per-site scale must then store zeros
    (1/max would overflow and turn exact zeros into NaN)."""
    shape = (4, 4, 4, 128)
    rng = np.random.default_rng(9)
    U = W.hot_links(rng, shape, 1, 0.2)
    bc = (1, 1, 1, -1)
    m = -0.2962963
    ctx = WilsonContext(shape, bc=bc)
    gauge = ctx.gauge(torch.from_numpy(U[0]))
    eta = np.zeros((2, *shape, 4, 3), dtype=np.complex128)
    eta[0, 0, 0, 0, 0, 0, 0] = 1.0
    eta[1, 0, 0, 0, 0, 3, 2] = 1.0
    b = ctx.apply("SCHUR_E_DAG", gauge, m, torch.from_numpy(eta), normalized=True)
    x, st = ctx.solve(gauge, b, m, op="eo_normal", tol=1e-10, maxiter=3000, inner="half")
    assert all(s["status"] == 2 for s in st), st
    bn, xn = b.cpu().numpy(), x.cpu().numpy()
    for r in range(2):
        s = W.schur_even(U, xn[r][None], m, bc, normalized=True)
        Ax = W.schur_even(U, s, m, bc, normalized=True, dag=True)[0]
        assert np.linalg.norm(bn[r] - Ax) / np.linalg.norm(bn[r]) <= 1e-10


@pytest.mark.parametrize("kappa", [0.12, 0.135])
@pytest.mark.parametrize("src", ["gauss", "point"])
def test_fp32_D_within_1e6(setup, kappa, src):
    """D and D^dag in FP32 (FP32 storage, 12-real FP32 links, FP32 arithmetic)
    against the FP64 oracle at 1e-6 relative, at both masses of the measured
    configurations and on a complex boundary phase as well as the antiperiodic one."""
    shape, U, bc, ctx, gauge = setup
    m = W.kappa_to_mass(kappa)
    x = _fields(shape, 3)[src]
    for c, g, b in ((ctx, gauge, bc), *_phase_ctx(shape, U)):
        eng = Engine(c, g, 1, op="normal", inner="single")
        d = eng.debug_apply(3, m, torch.from_numpy(x)).cpu().numpy()
        dd = eng.debug_apply(5, m, torch.from_numpy(x)).cpu().numpy()
        eng.close()
        assert rel(d, W.apply_D(U, x[None], m, b)[0]) < 1e-6, (kappa, src, b)
        assert rel(dd, W.apply_Ddag(U, x[None], m, b)[0]) < 1e-6, (kappa, src, b)


def _phase_ctx(shape, U):
    bc = (1, 1, complex(np.cos(np.pi / 3), np.sin(np.pi / 3)), -1)
    ctx = WilsonContext(shape, bc=bc)
    return [(ctx, ctx.gauge(torch.from_numpy(U[0])), bc)]


def test_fp16_hop_with_fp32_colour_multiply():
    """The FP16 engines multiply by the links in packed FP16 by default; the FP32-pair colour
    multiply (WL_HALF_COLOR=0, kept for comparisons; the choice is read once per process)
    must meet the same FP16 bounds, checked in a child process."""
    import os
    import subprocess
    import sys

    from tests.conftest import ROOT

    code = ("import tests.test_gpu_sloppy as T, numpy as np, torch\n"
            "from oracle import wilson as W\n"
            "shape = (4, 4, 4, 8); rng = np.random.default_rng(7); U = W.hot_links(rng, shape, 1, 0.2)\n"
            "ctx = T.WilsonContext(shape, bc=(1, 1, 1, -1)); g = ctx.gauge(torch.from_numpy(U[0]))\n"
            "m = -0.2962963; eng = T.Engine(ctx, g, 1, op='eo_normal', inner='half')\n"
            "for src, x in T._fields(shape, 1).items():\n"
            "    xe = W.project(x[None], 0)\n"
            "    ref = W.schur_even(U, W.schur_even(U, xe, m, (1, 1, 1, -1), normalized=True), m, (1, 1, 1, -1),"
            " normalized=True, dag=True)\n"
            "    out = eng.debug_apply(2, m, torch.from_numpy(xe[0])).cpu().numpy()\n"
            "    assert T.rel(out, ref[0]) < T.TOLS['half'], (src, T.rel(out, ref[0]))\n"
            "print('fp32 colour ok')\n")
    env = dict(os.environ, WL_HALF_COLOR="0")
    res = subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=env, capture_output=True, text=True,
                         timeout=600)
    assert res.returncode == 0 and "fp32 colour ok" in res.stdout, res.stdout[-2000:] + res.stderr[-4000:]


def test_fp16_lanes_hop_with_fp32_accumulation():
    """The 16-lane FP16 hop sums its eight contributions in packed FP16 by default; the FP32
    accumulation form (WL_HALF_ACC=0, kept for comparisons; read once per process) must meet
    the same FP16 operator bound and solve 16 RHS to an FP64 true residual <= 1e-10, checked
    in a child process."""
    import os
    import subprocess
    import sys

    from tests.conftest import ROOT

    code = ("import os, tests.test_gpu_sloppy as T, numpy as np, torch\n"
            "from oracle import wilson as W\n"
            "shape = (4, 4, 4, 8); bc = (1, 1, 1, -1); rng = np.random.default_rng(8)\n"
            "U = W.hot_links(rng, shape, 1, 0.2)\n"
            "ctx = T.WilsonContext(shape, bc=bc); g = ctx.gauge(torch.from_numpy(U[0]))\n"
            "m = -0.2962963; os.environ['WL_FORCE_TUNE'] = '1,128,1,16'\n"
            "eng = T.Engine(ctx, g, 16, op='eo_normal', inner='half', tol=1e-10, maxiter=3000)\n"
            "for src, x in T._fields(shape, 1).items():\n"
            "    xe = W.project(x[None], 0)\n"
            "    ref = W.schur_even(U, W.schur_even(U, xe, m, bc, normalized=True), m, bc, normalized=True, dag=True)\n"
            "    out = eng.debug_apply(2, m, torch.from_numpy(xe[0])).cpu().numpy()\n"
            "    assert T.rel(out, ref[0]) < T.TOLS['half'], (src, T.rel(out, ref[0]))\n"
            "b = W.project(W.gaussian_spinor(rng, shape, 16), 0)\n"
            "eng.admit(np.arange(16), torch.from_numpy(b), np.full(16, m))\n"
            "na = 16\n"
            "while na:\n"
            "    eng.step(8); _, na = eng.poll()\n"
            "for r in range(16):\n"
            "    xr, st = eng.retire(r); xr = xr.cpu().numpy()[None]\n"
            "    ax = W.schur_even(U, W.schur_even(U, xr, m, bc, normalized=True), m, bc, normalized=True, dag=True)[0]\n"
            "    assert st['status'] == 2 and np.linalg.norm(b[r] - ax) / np.linalg.norm(b[r]) <= 1e-10, (r, st)\n"
            "print('fp32 accumulation ok')\n")
    env = dict(os.environ, WL_HALF_ACC="0")
    res = subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=env, capture_output=True, text=True,
                         timeout=600)
    assert res.returncode == 0 and "fp32 accumulation ok" in res.stdout, res.stdout[-2000:] + res.stderr[-4000:]
