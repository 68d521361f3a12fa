"""Host-side logic without a GPU: the multi-rank aggregation of bench.py over
gloo (world size 2) and the serving loop's admission / continuous batching
with fake engines standing in for the device solver."""

import math
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bench
from jaxqft_b200 import serving


# --------------------------------------------------------------------------- bench over 2 gloo ranks
def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, t_local, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t_max, value = bench.aggregate_over_ranks(t_local[rank], 16, dist, torch.device("cpu"))
        out[rank] = (t_max, value)
    finally:
        dist.destroy_process_group()


def test_bench_value_is_world_units_over_max_rank_time():
    world, port = 2, _free_port()
    t_local = [0.25, 0.40]
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(world, port, t_local, out), nprocs=world, join=True)
        res = dict(out)
    for r in range(world):
        t_max, value = res[r]
        assert t_max == pytest.approx(0.40)
        assert value == pytest.approx(world * 16 / 0.40)


def test_bench_single_rank_aggregation():
    t_max, value = bench.aggregate_over_ranks(0.5, 16)
    assert t_max == 0.5 and value == pytest.approx(32.0)


# --------------------------------------------------------------------------- serving with fake engines
class FakeCtx:
    def __init__(self, vol, engine_bytes):
        self.vol, self._bytes = vol, engine_bytes

    def engine_bytes(self, op, inner, nslots):
        return self._bytes

    def apply(self, op, gauge, mass, eta, normalized=True):
        return eta.clone()


class FakeEngine:
    """Slots converge `solve_steps` iterations (step() calls of one iteration) after their
    admission; run() iterates until a slot finishes."""

    solve_steps = 3
    created = []

    def __init__(self, ctx, gauge, nslots, op, inner, tol, maxiter):
        self.nslots = nslots
        self.left = {}
        self.closed = False
        self.max_busy = 0
        FakeEngine.created.append(self)

    def admit(self, slots, b, masses, tols=None):
        assert not self.closed
        for s in slots:
            assert s not in self.left, "slot admitted twice"
            self.left[int(s)] = self.solve_steps
        self.max_busy = max(self.max_busy, len(self.left))

    def step(self, n):
        for s in self.left:
            self.left[s] = max(0, self.left[s] - 1)

    def run(self, n):
        # as wl_engine_run: steps until a running slot finishes, at most n
        self.run_caps = getattr(self, "run_caps", []) + [n]
        for _ in range(n):
            running = [s for s, k in self.left.items() if k > 0]
            if not running:
                break
            self.step(1)
            if any(self.left[s] == 0 for s in running):
                break

    def poll(self):
        st = np.zeros(self.nslots, dtype=np.int32)
        for s, k in self.left.items():
            st[s] = serving.L.SLOT_CONVERGED if k == 0 else 1
        return st, sum(1 for k in self.left.values() if k > 0)

    def poll_async(self):
        # the copies "land" on the second readiness check: the loop must cope with a poll in flight
        self._snap, self._checks = self.poll(), 0

    def poll_ready(self):
        self._checks += 1
        return self._snap if self._checks >= 2 else None

    def retire(self, s, out=None):
        assert self.left.pop(s) == 0
        return out, {"iters": 10, "status": serving.L.SLOT_CONVERGED, "true_res": 1e-11, "reliable_updates": 1}

    def close(self):
        self.closed = True


def make_server(volumes, nslots, budget, engine_bytes):
    srv = object.__new__(serving.PropagatorServer)
    srv.device = torch.device("cpu")
    srv.nslots, srv.inner, srv.tol, srv.maxiter, srv.iters_per_poll = nslots, "half", 1e-10, 100, 8
    srv.run_cap, srv.device_runs = 256, True
    srv.keep_solutions = True
    srv.hbm_budget = budget
    srv.ctx = {v: FakeCtx(v, engine_bytes) for v in volumes}
    srv.gauges = {(v, s): object() for v in volumes for s in range(2)}
    srv.resident_bytes = 0
    srv.engines, srv.engine_bytes, srv.peak_engine_bytes = {}, 0, 0
    srv.queue = serving.collections.deque()
    srv.done = []
    return srv


class FakeClock:
    def __init__(self, dt):
        self.t, self.dt = 0.0, dt

    def __call__(self):
        self.t += self.dt
        return self.t


@pytest.fixture
def fake_engines(monkeypatch):
    FakeEngine.created = []
    monkeypatch.setattr(serving.L, "Engine", FakeEngine)
    monkeypatch.setattr(serving.time, "sleep", lambda s: None)
    return FakeEngine


VOL = (4, 4, 4, 4)


def test_serving_budget_admits_one_engine_at_a_time(fake_engines):
    srv = make_server([VOL], nslots=8, budget=150, engine_bytes=100)
    reqs = [serving.Request(rid=i, volume=VOL, gauge=i % 2, kappa=0.125, nrhs=2, kind="point", t_arrive=0.0)
            for i in range(4)]
    done = srv.run(reqs, time_fn=FakeClock(1e-3))
    assert sorted(r.rid for r in done) == [0, 1, 2, 3]
    assert srv.peak_engine_bytes <= 150
    assert len(fake_engines.created) >= 2  # the idle engine of gauge 0 was released for gauge 1
    assert all(e.closed for e in fake_engines.created[:-1])
    for r in done:
        assert r.t_done >= r.t_arrive and r.latency_ms >= 0
        assert len(r.stats) == r.nrhs and all(s["status"] == serving.L.SLOT_CONVERGED for s in r.stats)


def test_serving_continuous_batching_shares_an_engine(fake_engines):
    srv = make_server([VOL], nslots=8, budget=10**9, engine_bytes=100)
    # same gauge: the second request joins the engine while the first is mid-solve
    reqs = [serving.Request(rid=0, volume=VOL, gauge=0, kappa=0.125, nrhs=5, kind="point", t_arrive=0.0),
            serving.Request(rid=1, volume=VOL, gauge=0, kappa=0.130, nrhs=3, kind="gaussian", t_arrive=0.0015,
                            seed=7)]
    done = srv.run(reqs, time_fn=FakeClock(1e-3))
    assert len(done) == 2 and len(fake_engines.created) == 1
    assert fake_engines.created[0].max_busy == 8
    summ = serving.summarize(done, wall=1.0)
    assert summ["solves"] == 8 and summ["all_converged"] and summ["requests"] == 2


def test_serving_trace_and_queue_summary(fake_engines):
    srv = make_server([VOL], nslots=4, budget=10**9, engine_bytes=100)
    reqs = [serving.Request(rid=i, volume=VOL, gauge=0, kappa=0.125, nrhs=3, kind="point", t_arrive=0.0)
            for i in range(3)]
    srv.run(reqs, time_fn=FakeClock(1e-2))
    assert srv.trace and srv.trace[0][1] >= 1  # requests queued at the start
    q = serving.queue_summary(srv.trace, arrival_window=0.0, points=5)
    assert q["max_queued"] >= 1 and len(q["samples"]) <= 5
    assert serving.queue_summary([], 1.0)["max_queued"] == 0


def test_serving_releases_finished_requests_buffers(fake_engines):
    srv = make_server([VOL], nslots=8, budget=10**9, engine_bytes=100)
    srv.keep_solutions = False
    reqs = [serving.Request(rid=i, volume=VOL, gauge=0, kappa=0.125, nrhs=2, kind="point", t_arrive=0.0)
            for i in range(3)]
    done = srv.run(reqs, time_fn=FakeClock(1e-3))
    assert len(done) == 3 and all(r.x is None and r.b is None and r.eta is None for r in done)
    assert all(len(r.stats) == 2 for r in done)


def test_serving_waits_for_free_slots(fake_engines):
    srv = make_server([VOL], nslots=4, budget=10**9, engine_bytes=100)
    reqs = [serving.Request(rid=i, volume=VOL, gauge=0, kappa=0.125, nrhs=3, kind="point", t_arrive=0.0)
            for i in range(3)]
    done = srv.run(reqs, time_fn=FakeClock(1e-3))
    assert [r.rid for r in done] == [0, 1, 2]  # one at a time: 3 + 3 > 4 slots
    assert fake_engines.created[0].max_busy == 3


def test_serving_rejects_requests_larger_than_an_engine(fake_engines):
    srv = make_server([VOL], nslots=4, budget=10**9, engine_bytes=100)
    req = serving.Request(rid=0, volume=VOL, gauge=0, kappa=0.125, nrhs=5, kind="point", t_arrive=0.0)
    with pytest.raises(ValueError):
        srv.run([req], time_fn=FakeClock(1e-3))


def test_poisson_requests_statistics():
    reqs = serving.poisson_requests(50.0, 200.0, [(8, 8, 8, 8), (12, 12, 12, 24)], seed=3)
    assert abs(len(reqs) / 200.0 - 50.0) < 3.0
    t = np.array([r.t_arrive for r in reqs])
    assert np.all(np.diff(t) > 0)
    k = np.array([r.kappa for r in reqs])
    n = np.array([r.nrhs for r in reqs])
    assert k.min() >= 0.120 and k.max() <= 0.135 and n.min() == 1 and n.max() == 12
    assert math.isclose(np.mean([r.kind == "point" for r in reqs]), 0.5, abs_tol=0.05)


def test_serving_run_caps_scale_with_volume(fake_engines):
    """Device-side runs are capped at iters_per_poll on the largest served volume and at
    proportionally more iterations on smaller ones (a similar wall time per run), within
    [iters_per_poll, run_cap]; host-stepped mode calls step() instead."""
    big, small = (8, 8, 8, 8), (4, 4, 4, 4)  # 16x fewer sites
    srv = make_server([big, small], nslots=4, budget=10**9, engine_bytes=100)
    assert srv.run_iters(big) == 8 and srv.run_iters(small) == 128
    srv.run_cap = 64
    assert srv.run_iters(small) == 64
    reqs = [serving.Request(rid=0, volume=big, gauge=0, kappa=0.125, nrhs=2, kind="point", t_arrive=0.0),
            serving.Request(rid=1, volume=small, gauge=0, kappa=0.125, nrhs=2, kind="point", t_arrive=0.0)]
    done = srv.run(reqs, time_fn=FakeClock(1e-3))
    assert len(done) == 2
    caps = {tuple(sorted(set(e.run_caps))) for e in fake_engines.created}
    assert caps == {(8,), (64,)}
    srv.device_runs = False
    srv.done = []
    before = len(fake_engines.created)
    reqs = [serving.Request(rid=2, volume=big, gauge=1, kappa=0.125, nrhs=1, kind="point", t_arrive=0.0)]
    done = srv.run(reqs, time_fn=FakeClock(1e-3))
    assert len(done) == 1
    assert not hasattr(fake_engines.created[before], "run_caps")  # stepped, never run

