"""Continuous-batching propagator-solve server on one B200.

Requests ask for Wilson propagator columns: for each of their RHS (point
sources at site 0 or Gaussian spinors) solve the even-odd normal system
(M^dag M) x = M^dag eta on one of the resident gauge fields, at the request's
own kappa, to an FP64 true residual <= tol.  This is the solve pattern of
jaxqft/core/measurements.py:277-372 (sources passed through the adjoint, then
a normal-equation CG), batched across requests.

* Gauge fields stay resident in HBM (per volume, one per seed).
* One solver engine (``wl_engine``) per (volume, gauge field) holds a fixed set
  of RHS slots with per-slot kappa/tolerance; a request is admitted into free
  slots while other slots of the same engine are mid-solve, and its slots are
  retired (and freed) as they converge -- continuous batching at RHS level.
* Engines are created on demand while the sum of their device footprints
  (``wl_engine_bytes``) stays under the HBM budget; requests that do not fit
  wait in a FIFO queue.  Each engine runs on its own CUDA stream, so work for
  different volumes / gauge fields overlaps on the device.
* Latency = completion - arrival (queueing included), measured on the host
  clock; each response's solution stays in device memory.
* A request with ``measure="pion"`` (12 point sources) also gets the pion
  two-point function (jaxqft/core/measurements.py:375-390) of its propagator:
  the odd sites are reconstructed from the even solution
  (x_e = M^-1 eta_e / m0, x_o = -(K x_e)_o / m0, su3_wilson_nf2.py:1325-1335)
  and contracted on the device.
"""

from __future__ import annotations

import collections
import math
import time
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np
import torch

from . import lib as L


@dataclass
class Request:
    rid: int
    volume: Tuple[int, ...]
    gauge: int
    kappa: float
    nrhs: int
    kind: str  # "point" | "gaussian"
    t_arrive: float
    seed: int = 0
    t_admit: Optional[float] = None
    t_done: Optional[float] = None
    slots: List[int] = field(default_factory=list)
    eta: Optional[torch.Tensor] = None
    b: Optional[torch.Tensor] = None
    x: Optional[torch.Tensor] = None
    stats: List[dict] = field(default_factory=list)
    pending: int = 0
    measure: Optional[str] = None      # "pion": contract the 12 point-source columns
    pion: Optional[np.ndarray] = None  # C(dt), dt = 0..Lt-1, when measured

    @property
    def mass(self) -> float:
        return 1.0 / (2.0 * self.kappa) - 4.0

    @property
    def latency_ms(self) -> float:
        return (self.t_done - self.t_arrive) * 1e3


def make_sources(req: Request, device) -> torch.Tensor:
    """Raw sources eta for a request: point sources delta(x,0) delta(s,c; k)
    for k = 0..nrhs-1 (spin x colour), or complex Gaussians with E|z|^2 = 1."""
    eta = torch.zeros((req.nrhs, *req.volume, 4, 3), dtype=torch.complex128, device=device)
    if req.kind == "point":
        for k in range(req.nrhs):
            eta[k, 0, 0, 0, 0, (k % 12) // 3, k % 3] = 1.0
    else:
        g = torch.Generator(device=device)
        g.manual_seed(int(req.seed))
        shp = eta.shape
        eta = torch.complex(torch.randn(shp, generator=g, device=device, dtype=torch.float64),
                            torch.randn(shp, generator=g, device=device, dtype=torch.float64)) / math.sqrt(2.0)
    return eta


def even_mask(volume, device) -> torch.Tensor:
    par = torch.zeros(volume, dtype=torch.int64, device=device)
    for ax, n in enumerate(volume):
        shp = [1] * 4
        shp[ax] = n
        par = par + torch.arange(n, device=device).reshape(shp)
    return (par % 2 == 0).to(torch.complex128)[..., None, None]


class _Slotted:
    """An engine plus slot bookkeeping."""

    def __init__(self, engine: L.Engine, nslots: int, nbytes: int):
        self.engine = engine
        self.nslots = nslots
        self.nbytes = nbytes
        self.owner: Dict[int, Tuple[Request, int]] = {}  # slot -> (request, rhs index)

    @property
    def free(self) -> int:
        return self.nslots - len(self.owner)

    def free_slots(self, k: int) -> List[int]:
        return [s for s in range(self.nslots) if s not in self.owner][:k]


class PropagatorServer:
    def __init__(self, volumes: Sequence[Tuple[int, ...]], gauge_seeds: Sequence[int] = (0, 1, 2, 3),
                 link_scale: float = 0.2, nslots: int = 16, inner: str = "half", tol: float = 1e-10,
                 maxiter: int = 4000, hbm_budget_bytes: Optional[int] = None, iters_per_poll: int = 8,
                 run_cap: int = 256, device_runs: bool = True, device=None, keep_solutions: bool = True):
        if not torch.cuda.is_available():
            raise RuntimeError("the serving loop requires a CUDA device")
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.nslots, self.inner, self.tol, self.maxiter = int(nslots), inner, float(tol), int(maxiter)
        self.iters_per_poll = int(iters_per_poll)
        self.run_cap = int(run_cap)
        # False: step each engine by iters_per_poll iterations per poll (wl_engine_step), for
        # comparisons
        self.device_runs = bool(device_runs)
        # False: a finished request's device buffers (sources, right-hand sides, solutions) are
        # released as soon as it completes, as a server does once the response has been sent;
        # only its statistics (and its pion correlator) are kept
        self.keep_solutions = bool(keep_solutions)
        free, total = torch.cuda.mem_get_info(self.device)
        self.hbm_budget = int(hbm_budget_bytes) if hbm_budget_bytes is not None else int(0.6 * free)
        self.ctx: Dict[Tuple[int, ...], L.WilsonContext] = {}
        self.gauges: Dict[Tuple[Tuple[int, ...], int], L.Gauge] = {}
        self.resident_bytes = 0
        for vol in volumes:
            vol = tuple(int(v) for v in vol)
            self.ctx[vol] = L.WilsonContext(vol, bc=(1, 1, 1, -1), device=self.device)
            for seed in gauge_seeds:
                U = self._hot_links(vol, link_scale, seed)
                self.gauges[(vol, int(seed))] = self.ctx[vol].gauge(U)
                self.resident_bytes += int(np.prod(vol)) * 4 * 9 * 16 * 2 + int(np.prod(vol)) * 4 * 9 * 16
                del U
        self.engines: Dict[Tuple[Tuple[int, ...], int], _Slotted] = {}
        self.engine_bytes = 0
        self.peak_engine_bytes = 0
        self.queue: collections.deque = collections.deque()
        self.done: List[Request] = []

    def _hot_links(self, vol, scale, seed):
        g = torch.Generator(device=self.device)
        g.manual_seed(int(seed))
        shp = (4, *vol, 3, 3)
        a = scale * torch.complex(torch.randn(shp, generator=g, device=self.device, dtype=torch.float64),
                                  torch.randn(shp, generator=g, device=self.device, dtype=torch.float64))
        y = 0.5 * (a - a.conj().transpose(-1, -2))
        tr = torch.diagonal(y, dim1=-2, dim2=-1).sum(-1) / 3.0
        y = y - tr[..., None, None] * torch.eye(3, dtype=y.dtype, device=self.device)
        return torch.linalg.matrix_exp(y)

    # ------------------------------------------------------------------ admission
    def _engine_for(self, req: Request) -> Optional[_Slotted]:
        key = (req.volume, req.gauge)
        if key in self.engines:
            return self.engines[key]
        ctx = self.ctx[req.volume]
        nbytes = ctx.engine_bytes("eo_normal", self.inner, self.nslots)
        if self.engine_bytes + nbytes > self.hbm_budget:
            # release an idle engine to make room, if any
            for k, e in list(self.engines.items()):
                if not e.owner:
                    e.engine.close()
                    self.engine_bytes -= e.nbytes
                    del self.engines[k]
                    if self.engine_bytes + nbytes <= self.hbm_budget:
                        break
        if self.engine_bytes + nbytes > self.hbm_budget:
            return None
        eng = L.Engine(ctx, self.gauges[key], self.nslots, op="eo_normal", inner=self.inner, tol=self.tol,
                       maxiter=self.maxiter)
        se = _Slotted(eng, self.nslots, nbytes)
        self.engines[key] = se
        self.engine_bytes += nbytes
        self.peak_engine_bytes = max(self.peak_engine_bytes, self.engine_bytes)
        return se

    def _admit(self, req: Request, se: _Slotted, now: float) -> None:
        ctx, gauge = self.ctx[req.volume], self.gauges[(req.volume, req.gauge)]
        eta = make_sources(req, self.device) * even_mask(req.volume, self.device)
        # b = M^dag eta_e on the engine's own stream ordering (ctx stream, then engine waits)
        req.b = ctx.apply("SCHUR_E_DAG", gauge, req.mass, eta, normalized=True)
        req.slots = se.free_slots(req.nrhs)
        for i, s in enumerate(req.slots):
            se.owner[s] = (req, i)
        req.x = torch.empty_like(req.b)
        req.stats = [None] * req.nrhs
        req.pending = req.nrhs
        se.engine.admit(req.slots, req.b, np.full(req.nrhs, req.mass), tols=np.full(req.nrhs, self.tol))
        req.t_admit = now

    def _try_admit(self, now: float) -> None:
        waiting = collections.deque()
        while self.queue:
            req = self.queue.popleft()
            if req.nrhs > self.nslots:
                raise ValueError(f"request {req.rid}: {req.nrhs} RHS exceed the {self.nslots} slots of an engine")
            se = self._engine_for(req)
            if se is not None and se.free >= req.nrhs:
                self._admit(req, se, now)
            else:
                waiting.append(req)
        self.queue = waiting

    # ------------------------------------------------------------------ main loop
    def run(self, requests: Sequence[Request], time_fn=time.perf_counter) -> List[Request]:
        """Serve `requests` (arrival times in seconds from the start).

        The host never waits on one engine while another could work: every busy
        engine with nothing in flight gets one device-side run of CG iterations
        (wl_engine_run: it stops by itself as soon as one of its slots finishes) and
        a non-blocking status poll on its own stream (wl_engine_poll_async); the
        loop then admits arrivals, and handles each engine whose poll has landed
        (wl_engine_poll_ready) by retiring its converged slots and starting its next
        run.  A run is capped at about the time of `iters_per_poll` iterations on the
        largest served volume (`run_iters`), because a request admitted into an
        engine starts iterating only when the engine's current run ends.
        `self.trace` samples (seconds, queued requests, busy slots)."""
        pending = collections.deque(sorted(requests, key=lambda r: r.t_arrive))
        t0 = time_fn()
        inflight = set()
        self.trace = []
        next_sample = 0.0
        while pending or self.queue or inflight or any(e.owner for e in self.engines.values()):
            now = time_fn() - t0
            while pending and pending[0].t_arrive <= now:
                self.queue.append(pending.popleft())
            if self.queue:
                self._try_admit(now)
            for key, e in self.engines.items():
                if e.owner and key not in inflight:
                    if self.device_runs:
                        e.engine.run(self.run_iters(key[0]))
                    else:
                        e.engine.step(self.iters_per_poll)
                    e.engine.poll_async()
                    inflight.add(key)
            landed = False
            for key in list(inflight):
                e = self.engines[key]
                r = e.engine.poll_ready()
                if r is None:
                    continue
                inflight.discard(key)
                landed = True
                st, _ = r
                for s in list(e.owner):
                    if st[s] >= L.SLOT_CONVERGED:
                        req, i = e.owner.pop(s)
                        _, info = e.engine.retire(s, out=req.x[i])
                        req.stats[i] = info
                        req.pending -= 1
                        if req.pending == 0:
                            if req.measure == "pion":
                                self._measure_pion(req)
                            req.t_done = time_fn() - t0
                            if not self.keep_solutions:
                                req.eta = req.b = req.x = None
                            self.done.append(req)
            if now >= next_sample:
                self.trace.append((now, len(self.queue), sum(len(e.owner) for e in self.engines.values())))
                next_sample = now + 0.05
            if not landed:
                if not inflight and pending:
                    time.sleep(max(0.0, min(pending[0].t_arrive - (time_fn() - t0), 0.01)))
                else:
                    time.sleep(5e-5)  # the device is working; check again shortly
        if self.device.type == "cuda":
            torch.cuda.synchronize(self.device)
        return self.done

    def run_iters(self, volume) -> int:
        """Iteration cap of one device-side run on `volume`: iters_per_poll scaled by the
        largest served volume over this one (an iteration's time grows with the volume),
        between iters_per_poll and run_cap."""
        vmax = max(int(np.prod(v)) for v in self.ctx)
        scaled = self.iters_per_poll * vmax // max(1, int(np.prod(volume)))
        return int(max(self.iters_per_poll, min(self.run_cap, scaled)))

    def _measure_pion(self, req: Request) -> None:
        if req.kind != "point" or req.nrhs != 12:
            raise ValueError(f"request {req.rid}: the pion measurement needs the 12 point sources")
        ctx, gauge = self.ctx[req.volume], self.gauges[(req.volume, req.gauge)]
        m0 = req.mass + 4.0
        even = even_mask(req.volume, self.device)
        xe = req.x * even / m0
        kxe = ctx.apply("D", gauge, req.mass, xe) - m0 * xe
        prop = xe - kxe * (1.0 - even) / m0
        req.pion = ctx.pion_correlator(prop, 0)

    def close(self):
        for e in self.engines.values():
            e.engine.close()
        self.engines.clear()


def poisson_requests(rate: float, duration: float, volumes, kappa_range=(0.120, 0.135), max_rhs: int = 12,
                     ngauge: int = 4, seed: int = 0) -> List[Request]:
    """Poisson arrivals (mean `rate` per second) over `duration` seconds with
    volume, kappa, RHS count and source kind drawn uniformly."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t > duration:
            break
        vol = tuple(volumes[rng.integers(len(volumes))])
        out.append(Request(rid=len(out), volume=vol, gauge=int(rng.integers(ngauge)),
                           kappa=float(rng.uniform(*kappa_range)), nrhs=int(rng.integers(1, max_rhs + 1)),
                           kind="point" if rng.random() < 0.5 else "gaussian", t_arrive=t,
                           seed=int(rng.integers(1 << 30))))
    return out


def queue_summary(trace, arrival_window: float, points: int = 40) -> dict:
    """Queue length over time from PropagatorServer.trace: the largest queue, the
    queue when arrivals stop, and up to `points` (seconds, queued, busy slots) samples."""
    if not trace:
        return {"max_queued": 0, "queued_at_window_end": 0, "samples": []}
    t = np.array([s[0] for s in trace])
    q = np.array([s[1] for s in trace])
    k = int(np.searchsorted(t, arrival_window, side="right")) - 1
    pick = np.unique(np.linspace(0, len(trace) - 1, min(points, len(trace))).astype(int))
    return {"max_queued": int(q.max()), "queued_at_window_end": int(q[max(k, 0)]),
            "samples": [[round(float(trace[i][0]), 3), int(trace[i][1]), int(trace[i][2])] for i in pick]}


def summarize(done: Sequence[Request], wall: float) -> dict:
    lat = np.array([r.latency_ms for r in done])
    nsol = sum(r.nrhs for r in done)
    res = max((s["true_res"] for r in done for s in r.stats), default=0.0)
    conv = all(s["status"] == L.SLOT_CONVERGED for r in done for s in r.stats)
    per_vol = {}
    for vol in sorted({r.volume for r in done}, key=lambda v: int(np.prod(v))):
        lv = np.array([r.latency_ms for r in done if r.volume == vol])
        per_vol["x".join(map(str, vol))] = {"requests": int(lv.size), "p50_ms": float(np.percentile(lv, 50)),
                                            "p99_ms": float(np.percentile(lv, 99))}
    return {"requests": len(done), "solves": nsol, "wall_s": wall, "solves_per_s": nsol / wall if wall > 0 else 0.0,
            "p50_ms": float(np.percentile(lat, 50)) if len(lat) else None,
            "p99_ms": float(np.percentile(lat, 99)) if len(lat) else None,
            "mean_ms": float(lat.mean()) if len(lat) else None, "max_true_res": res, "all_converged": conv,
            "per_volume": per_vol}


VOLUMES = [(8, 8, 8, 8), (12, 12, 12, 24), (16, 16, 16, 32), (24, 24, 24, 48)]


def serve_once(server: PropagatorServer, rate: float, seconds: float, seed: int = 1) -> dict:
    """One Poisson stream against a warm server: latency percentiles, throughput
    and the queue length over time (the queue at the end of the arrival window
    tells whether the rate is sustained)."""
    server.done = []
    reqs = poisson_requests(rate, seconds, VOLUMES, seed=seed)
    t0 = time.perf_counter()
    done = server.run(reqs)
    wall = time.perf_counter() - t0
    s = summarize(done, wall)
    last_arrival = max((r.t_arrive for r in reqs), default=0.0)
    last_done = max((r.t_done for r in done), default=0.0)
    s.update({"rate_per_s": rate, "arrival_window_s": seconds, "drain_s": max(0.0, last_done - last_arrival),
              "queue": queue_summary(server.trace, seconds)})
    return s


def warm_server(server: PropagatorServer, gauge_seeds=(0, 1, 2, 3)) -> None:
    """Server start-up: one 1-RHS request per (volume, gauge field) allocates,
    tunes and graph-captures every engine before any timed stream."""
    warm = [Request(rid=-1 - i, volume=tuple(v), gauge=g, kappa=0.125, nrhs=1, kind="gaussian", t_arrive=0.0,
                    seed=99 + i)
            for i, (v, g) in enumerate((v, g) for v in VOLUMES for g in gauge_seeds)]
    server.run(warm)
    server.done = []


def main(argv=None):
    """python -m jaxqft_b200.serving --rates 50 --seconds 30   (one JSON line per rate)"""
    import argparse
    import json

    ap = argparse.ArgumentParser(description="Poisson propagator-request streams against a warm server")
    ap.add_argument("--rates", default="50", help="comma-separated mean arrival rates (requests/s)")
    ap.add_argument("--seconds", type=float, default=30.0, help="arrival window per rate")
    ap.add_argument("--inner", default="half")
    ap.add_argument("--compare-runs", action="store_true",
                    help="serve each rate twice per seed, with device-side runs and host-stepped engines")
    ap.add_argument("--seeds", default="1", help="comma-separated request-stream seeds")
    args = ap.parse_args(argv)
    server = PropagatorServer(VOLUMES, gauge_seeds=(0, 1, 2, 3), nslots=16, inner=args.inner, keep_solutions=False)
    warm_server(server)
    modes = (True, False) if args.compare_runs else (True,)
    for seed in (int(x) for x in args.seeds.split(",")):
        for rate in (float(r) for r in args.rates.split(",")):
            for mode in modes:
                server.device_runs = mode
                s = serve_once(server, rate, args.seconds, seed=seed)
                print(json.dumps({"serve": True, "device_runs": mode, "seed": seed, **s}), flush=True)
    server.close()


if __name__ == "__main__":
    main()
