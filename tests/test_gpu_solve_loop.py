"""wl_solve runs a whole solve as one CUDA graph launch: a WHILE node around the captured
CG iteration, continued by its finalize kernel while any slot is active (and never more
than the iteration limit plus a few).  wl_engine_run uses the same loop, stopping as soon
as a slot finishes.  Their results must be the host-driven iteration's: the same kernels
in the same order, so bitwise the same solutions, iteration counts and statuses, for
converged solves and for solves stopped at maxiter, and for slots that converge at
different iterations."""

import numpy as np
import pytest

from oracle import wilson as W

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("CUDA device required", allow_module_level=True)

from jaxqft_b200.lib import SLOT_CONVERGED, SLOT_MAXITER, WilsonContext  # noqa: E402


@pytest.fixture(scope="module")
def setup():
    shape = (4, 4, 4, 8)
    rng = np.random.default_rng(77)
    U = W.hot_links(rng, shape, 1, 0.25)
    bc = (1, 1, 1, -1)
    ctx = WilsonContext(shape, bc=bc)
    gauge = ctx.gauge(torch.from_numpy(U[0]))
    return shape, U, bc, ctx, gauge, rng


@pytest.mark.parametrize("inner", ["double", "single", "half"])
@pytest.mark.parametrize("op", ["eo_normal", "normal"])
def test_loop_graph_equals_host_loop(setup, inner, op):
    shape, U, bc, ctx, gauge, rng = setup
    n = 3
    b = W.gaussian_spinor(rng, shape, n)
    b[1] *= 1e-3
    if op == "eo_normal":
        b = W.project(b, 0)
    masses = np.array([-0.2, 0.05, -0.1])
    xg, sg = ctx.solve(gauge, torch.from_numpy(b), masses, op=op, tol=1e-10, maxiter=2000, inner=inner)
    xh, sh = ctx.solve(gauge, torch.from_numpy(b), masses, op=op, tol=1e-10, maxiter=2000, inner=inner,
                       use_graph=False)
    assert torch.equal(xg, xh)
    for a, c in zip(sg, sh):
        assert a["status"] == c["status"] == SLOT_CONVERGED
        assert a["iters"] == c["iters"] and a["reliable_updates"] == c["reliable_updates"]
    for r in range(n):
        x = xg[r].cpu().numpy()[None]
        if op == "eo_normal":
            s = W.schur_even(U, x, masses[r], bc, normalized=True)
            ax = W.schur_even(U, s, masses[r], bc, normalized=True, dag=True)[0]
        else:
            ax = W.apply_normal(U, x, masses[r], bc)[0]
        assert np.linalg.norm(b[r] - ax) / np.linalg.norm(b[r]) <= 1e-10


def test_loop_graph_stops_at_maxiter(setup):
    shape, U, bc, ctx, gauge, rng = setup
    b = W.project(W.gaussian_spinor(rng, shape, 2), 0)
    masses = np.array([-0.3, -0.3])
    for it in (1, 7, 20):
        xg, sg = ctx.solve(gauge, torch.from_numpy(b), masses, tol=1e-12, maxiter=it, inner="single")
        xh, sh = ctx.solve(gauge, torch.from_numpy(b), masses, tol=1e-12, maxiter=it, inner="single",
                           use_graph=False)
        assert torch.equal(xg, xh), it
        for a, c in zip(sg, sh):
            assert a["status"] == c["status"] == SLOT_MAXITER, (it, a, c)
            assert a["iters"] == c["iters"] == it, (it, a, c)


@pytest.mark.parametrize("inner,nslots", [("half", 4), ("single", 2)])
def test_engine_run_stops_when_a_slot_finishes(setup, inner, nslots):
    """wl_engine_run keeps iterating on the device until a slot finishes: the first launch
    returns with exactly the fast slot done and the others still running, and driving the
    engine with run() gives bitwise the solutions and iteration counts of step()/poll()."""
    from jaxqft_b200.lib import Engine

    shape, U, bc, ctx, gauge, rng = setup
    masses = np.array([-0.25, 0.8, -0.1, 0.3])[:nslots]  # slot 1 (heavy) converges first
    b = W.project(W.gaussian_spinor(rng, shape, nslots), 0)
    out = {}
    for mode in ("step", "run"):
        eng = Engine(ctx, gauge, nslots, op="eo_normal", inner=inner, tol=1e-10, maxiter=3000)
        eng.admit(np.arange(nslots), torch.from_numpy(b), masses)
        na, first = nslots, None
        while na:
            if mode == "step":
                eng.step(8)
            else:
                eng.run(1000)
            st, na = eng.poll()
            if first is None:
                first = st.copy()
        res = [eng.retire(r) for r in range(nslots)]
        eng.close()
        out[mode] = (res, first)
    first = out["run"][1]
    assert first[1] == SLOT_CONVERGED and all(first[r] == 1 for r in range(nslots) if r != 1), first
    for r in range(nslots):
        (xs, ss), (xr, sr) = out["step"][0][r], out["run"][0][r]
        assert sr["status"] == ss["status"] == SLOT_CONVERGED, (r, ss, sr)
        assert sr["iters"] == ss["iters"], (r, ss, sr)
        assert torch.equal(xs, xr), r
        x = xr.cpu().numpy()[None]
        s = W.schur_even(U, x, masses[r], bc, normalized=True)
        ax = W.schur_even(U, s, masses[r], bc, normalized=True, dag=True)[0]
        assert np.linalg.norm(b[r] - ax) / np.linalg.norm(b[r]) <= 1e-10
