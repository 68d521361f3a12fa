"""Continuous-batching serving: requests of different volumes, kappas, RHS counts
and source kinds, arriving while others are on the GPU, must each come back
(a) converged to an FP64 true residual <= 1e-10 and (b) equal to the same solve
run alone: ||M^dag M (x_mix - x_alone)|| / ||b|| <= 2e-10 (both solutions meet
the 1e-10 bound) and relative difference <= 1e-6."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("CUDA device required", allow_module_level=True)

from jaxqft_b200 import lib as L  # noqa: E402
from jaxqft_b200.serving import PropagatorServer, Request, summarize  # noqa: E402

VOLS = [(4, 4, 4, 4), (4, 4, 4, 8), (6, 6, 6, 6)]


def _requests():
    rng = np.random.default_rng(4)
    reqs = []
    for i in range(14):
        reqs.append(Request(rid=i, volume=VOLS[i % 3], gauge=int(rng.integers(2)), kappa=float(rng.uniform(0.12, 0.135)),
                            nrhs=int(rng.integers(1, 7)), kind="point" if i % 2 else "gaussian",
                            t_arrive=0.002 * i, seed=100 + i))
    return reqs


def _check(server, done):
    for r in done:
        assert all(s["status"] == L.SLOT_CONVERGED for s in r.stats), (r.rid, r.stats)
        ctx, gauge = server.ctx[r.volume], server.gauges[(r.volume, r.gauge)]
        bn = torch.linalg.vector_norm(r.b.reshape(r.nrhs, -1), dim=1)
        Ax = ctx.apply("SCHUR_E_NORMAL", gauge, r.mass, r.x, normalized=True)
        res = torch.linalg.vector_norm((r.b - Ax).reshape(r.nrhs, -1), dim=1) / bn
        assert float(res.max()) <= 1e-10, (r.rid, res)
        x1, st = ctx.solve(gauge, r.b, r.mass, op="eo_normal", tol=1e-10, maxiter=4000, inner="double")
        d = ctx.apply("SCHUR_E_NORMAL", gauge, r.mass, r.x - x1, normalized=True)
        dres = torch.linalg.vector_norm(d.reshape(r.nrhs, -1), dim=1) / bn
        assert float(dres.max()) <= 2e-10, (r.rid, dres)
        rel = torch.linalg.vector_norm((r.x - x1).reshape(r.nrhs, -1), dim=1) / torch.linalg.vector_norm(
            x1.reshape(r.nrhs, -1), dim=1)
        assert float(rel.max()) <= 1e-6, (r.rid, rel)


def test_mixed_requests_equal_standalone_solves():
    server = PropagatorServer(VOLS, gauge_seeds=(0, 1), nslots=8, inner="half", tol=1e-10, iters_per_poll=4)
    reqs = _requests()
    done = server.run(reqs)
    assert len(done) == len(reqs)
    # requests overlapped on the device: some were admitted before earlier ones finished
    overlap = sum(1 for a in done for b in done if a is not b and a.t_admit < b.t_done and b.t_admit < a.t_done)
    assert overlap > 0
    _check(server, done)
    s = summarize(done, max(r.t_done for r in done))
    assert s["all_converged"] and s["p99_ms"] >= s["p50_ms"] > 0
    server.close()


def test_hbm_budget_queues_requests():
    """A budget that fits a single engine: requests for other (volume, gauge)
    pairs wait until it is idle, then everything completes correctly."""
    probe = L.WilsonContext(VOLS[2])
    one = probe.engine_bytes("eo_normal", "half", 8)
    server = PropagatorServer(VOLS, gauge_seeds=(0, 1), nslots=8, inner="half", tol=1e-10,
                              hbm_budget_bytes=int(one * 1.2))
    reqs = _requests()
    done = server.run(reqs)
    assert len(done) == len(reqs)
    assert server.peak_engine_bytes <= int(one * 1.2)
    _check(server, done)
    server.close()


def test_pion_request_matches_direct_measurement():
    """A 12-point-source request with measure="pion", served among other
    requests, returns the pion correlator of the full propagator (odd sites
    reconstructed): equal to the EO propagator of measurements.py solved alone
    in FP64 (1e-6 relative: both solutions meet a 1e-10 true residual)."""
    from jaxqft_b200 import measurements as M

    server = PropagatorServer(VOLS, gauge_seeds=(0, 1), nslots=16, inner="half", tol=1e-10, iters_per_poll=4)
    reqs = _requests()[:6]
    pion = Request(rid=99, volume=(6, 6, 6, 6), gauge=1, kappa=0.13, nrhs=12, kind="point", t_arrive=0.004,
                   measure="pion")
    done = server.run(reqs + [pion])
    assert len(done) == 7 and pion.pion is not None
    ctx, gauge = server.ctx[pion.volume], server.gauges[(pion.volume, 1)]
    eta = M.point_sources(pion.volume, (0, 0, 0, 0), ctx.device)
    x, st = M.propagator_columns(ctx, gauge, pion.mass, eta, method="eo", inner="double", tol=1e-12)
    ref = ctx.pion_correlator(x, 0)
    assert np.allclose(pion.pion, ref, rtol=1e-6, atol=0), (pion.pion, ref)
    # the full propagator solves D x = eta
    Dx = ctx.apply("D", gauge, pion.mass, x)
    assert float(torch.linalg.vector_norm(Dx - eta) / torch.linalg.vector_norm(eta)) < 1e-9
    server.close()
