#!/usr/bin/env python
"""Benchmark: batched mixed-precision Wilson CG solves/s on 24^3x48 (B200).

Workload (one "step"): the even-odd preconditioned Wilson normal system
(M^dag M) x_e = b_e of jaxQFT's solve_eop_even_normal on a 24^3x48 lattice,
kappa = 0.135 (bare mass 1/(2 kappa) - 4), antiperiodic time boundary,
links exp(i*0.2*H) per link (H traceless Hermitian, Gaussian entries), and
16 right-hand sides -- 12 point sources (one per spin x colour at site 0) and
4 Gaussian spinors, each passed through M^dag as the propagator code passes
its sources through D^dag.  All 16 are solved in ONE batched CG whose inner
operator runs in FP16 storage / FP32 arithmetic with FP64 reliable updates,
to an FP64 true residual ||b - M^dag M x|| / ||b|| <= 1e-10 for every RHS.

Reported: value = solves/s of that batched mixed solve (device time, CUDA
events on the solver stream, inputs resident in HBM), next to plain FP64 CG
(one RHS at a time) on the same systems; e2e = the same solve through the
public API from pinned host buffers with host<->device copies timed; the
roofline of the dominant kernel (the fused CG hop, the FP16 16-RHS stencil with
the CG update in its epilogue; the plain stencil beside it) measured live; the
Dslash bandwidth (FP64, 1 RHS) in the internal layout and in the reference
layout; and a CPU baseline (the C restatement of the reference's CG on the
host cores).

Data is synthetic (seeded); every working set is larger than the 126 MB L2.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from jaxqft_b200.wilson import WilsonDiracOperator  # noqa: E402  (pure Python: the flop counter)

DIRAC = WilsonDiracOperator()

SHAPE = (24, 24, 24, 48)
KAPPA = 0.135
KAPPA_LIGHT = 0.130  # the same batched solve timed at the second coupling of the 16-RHS config
MASS = 1.0 / (2.0 * KAPPA) - 4.0
BC = (1, 1, 1, -1)
LINK_SCALE = 0.2
NRHS = 16
TOL = 1e-10
METRIC = "CG solves/s 24^3x48 mixed vs FP64 @1e-10; Dslash HBM GB/s; serve p50/p99 ms"
WORKLOAD = ("EO-preconditioned Wilson normal-equation CG (solve_eop_even_normal), 24^3x48, kappa 0.135, "
            "antiperiodic t, links exp(i*0.2*H), 16 RHS (12 point sources at site 0 + 4 Gaussian) in one batched "
            "FP16/FP32 CG with FP64 reliable updates, true residual 1e-10")


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return float(p.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


def profile_traffic(key: str):
    """Per-launch DRAM bytes of the dominant kernel from a committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "roofline_traffic.txt")
    if not os.path.exists(path):
        return None
    for line in open(path):
        parts = line.split()
        if len(parts) >= 2 and parts[0] == key:
            return float(parts[1])
    return None


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = threading.Thread(target=self._run, daemon=True)

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                for line in out.stdout.strip().splitlines():
                    f = [v.strip() for v in line.split(",")]
                    if len(f) >= 9:
                        self.samples.append(f)
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[5 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


# --------------------------------------------------------------------------- inputs
def make_inputs(torch, device, seed: int):
    """Links exp(TA(a (G1 + i G2))) (= exp(i a H)) and the 16 raw sources."""
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    shp = (4, *SHAPE, 3, 3)
    A = LINK_SCALE * torch.complex(torch.randn(shp, generator=g, device=device, dtype=torch.float64),
                                   torch.randn(shp, generator=g, device=device, dtype=torch.float64))
    Y = 0.5 * (A - A.conj().transpose(-1, -2))
    del A
    tr = torch.diagonal(Y, dim1=-2, dim2=-1).sum(-1) / 3.0
    Y = Y - tr[..., None, None] * torch.eye(3, device=device, dtype=Y.dtype)
    U = torch.linalg.matrix_exp(Y)
    del Y
    eta = torch.zeros((NRHS, *SHAPE, 4, 3), dtype=torch.complex128, device=device)
    for k in range(12):  # point sources at site 0 (an even site)
        eta[k, 0, 0, 0, 0, k // 3, k % 3] = 1.0
    fshape = (NRHS - 12, *SHAPE, 4, 3)
    eta[12:] = torch.complex(torch.randn(fshape, generator=g, device=device, dtype=torch.float64),
                             torch.randn(fshape, generator=g, device=device, dtype=torch.float64)) / np.sqrt(2.0)
    return U, eta


def even_mask(torch, device):
    x = [torch.arange(n, device=device) for n in SHAPE]
    par = (x[0][:, None, None, None] + x[1][None, :, None, None] + x[2][None, None, :, None]
           + x[3][None, None, None, :]) % 2
    return (par == 0).to(torch.complex128)[..., None, None]


# --------------------------------------------------------------------------- our arm
def aggregate_over_ranks(t_local: float, units_per_rank: int, dist=None, device=None):
    """Whole-job throughput of independent replicas: every rank solved
    `units_per_rank` systems in `t_local` seconds (device time); the job time
    is the max over ranks and the value is world * units / that time."""
    import torch

    world = 1 if dist is None else dist.get_world_size()
    t_max = float(t_local)
    if dist is not None:
        tt = torch.tensor([t_max], device=device, dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_max = float(tt.item())
    return t_max, world * units_per_rank / t_max


def run_ours(args):
    import torch

    from jaxqft_b200 import lib as L

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    ctx = L.WilsonContext(SHAPE, bc=BC, device=dev)
    U, eta = make_inputs(torch, dev, seed=rank)
    gauge = ctx.gauge(U)
    # b_e = M^dag eta_e  (normalized Schur dagger, even sites)
    b = ctx.apply("SCHUR_E_DAG", gauge, MASS, eta * even_mask(torch, dev), normalized=True)
    torch.cuda.synchronize()

    eng = L.Engine(ctx, gauge, NRHS, op="eo_normal", inner=args.inner, tol=TOL, maxiter=4000, delta=args.delta)
    estream = eng.stream
    x = torch.empty_like(b)
    slots = np.arange(NRHS)

    def batched_solve(engine, bb, xx, n, mass=MASS):
        engine.admit(np.arange(n), bb, mass)
        na = n
        while na > 0:
            engine.step(8)
            st, na = engine.poll()
        stats = []
        for s in range(n):
            _, info = engine.retire(s, out=xx[s])
            stats.append(info)
        return stats

    def timed(fn, stream):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / 1e3, out

    # warm-up (graph capture, autotune, first-touch)
    for _ in range(args.warmup):
        stats = batched_solve(eng, b, x, NRHS)
    launches0 = L.kernel_launches()
    times, all_stats = [], []
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            t, stats = timed(lambda: batched_solve(eng, b, x, NRHS), estream)
            times.append(t)
            all_stats.append(stats)
    torch.cuda.synchronize()
    launches = L.kernel_launches() - launches0
    t_max, value = aggregate_over_ranks(float(np.mean(times)), NRHS, dist, dev)
    iters = [s["iters"] for s in all_stats[-1]]
    res = max(s["true_res"] for st in all_stats for s in st)
    conv = all(s["status"] == 2 for st in all_stats for s in st)

    # ---- the same 16-RHS batched solve at kappa 0.130 (sources through that M^dag), same links
    m_light = 1.0 / (2.0 * KAPPA_LIGHT) - 4.0
    b_light = ctx.apply("SCHUR_E_DAG", gauge, m_light, eta * even_mask(torch, dev), normalized=True)
    batched_solve(eng, b_light, x, NRHS, m_light)
    t_light, st_light = [], []
    for _ in range(max(2, args.steps // 2)):
        t, st = timed(lambda: batched_solve(eng, b_light, x, NRHS, m_light), estream)
        t_light.append(t)
        st_light.append(st)
    _, light_value = aggregate_over_ranks(float(np.mean(t_light)), NRHS, dist, dev)
    light = {"kappa": KAPPA_LIGHT, "solves_per_s": light_value, "steps": len(t_light),
             "iters_min": min(s["iters"] for s in st_light[-1]), "iters_max": max(s["iters"] for s in st_light[-1]),
             "max_true_res": max(s["true_res"] for st in st_light for s in st),
             "all_converged": all(s["status"] == 2 for st in st_light for s in st)}
    del b_light

    # ---- plain FP64 CG baseline: one RHS at a time, same systems
    eng64 = L.Engine(ctx, gauge, 1, op="eo_normal", inner="double", tol=TOL, maxiter=4000)
    batched_solve(eng64, b[12:13], x[12:13], 1)  # warm-up
    t64, it64 = 0.0, []
    n64 = NRHS if args.fp64_all else 4
    for r in range(NRHS - n64, NRHS):
        t, st = timed(lambda r=r: batched_solve(eng64, b[r:r + 1], x[r:r + 1], 1), eng64.stream)
        t64 += t
        it64.append(st[0]["iters"])
    fp64_sps = n64 / t64
    # the Dslash in the internal layout (the EO hop K_oe of that FP64 CG: SoA FP64 spinors, 18-real FP64
    # links, 1 RHS; 8 links + 2 spinors per target site), timed alone with CUDA events on the engine stream
    eng64.time_hop(reps=5)
    n_ms, n_bytes = eng64.time_hop(reps=50)
    dslash_native = {"kernel": "EO hop K_oe, internal SoA layout, FP64 (18-real links), 1 RHS (autotuned shape)",
                     "ms_per_launch": n_ms, "algorithmic_bytes_per_launch": n_bytes,
                     "achieved": n_bytes / (n_ms * 1e-3) / 1e9, "unit": "GB/s"}
    dslash_native["frac"] = dslash_native["achieved"] / peaks()[0]
    dslash_native["peak"] = peaks()[0]
    dslash_native.update(naive_rate(np.prod(SHAPE) // 2, 1, 192, 144, n_ms))
    dslash_native.update(ref_gflops(DIRAC.flops_per_site_dslash(3) * int(np.prod(SHAPE)) // 2, n_ms,
                                    "flops_per_site_dslash x Vh"))
    eng64.close()

    # ---- live rooflines of the FP16 16-RHS hops: the plain stencil (K_oe p) and, below, the dominant kernel
    hop_ms, hop_bytes = eng.time_hop(reps=20)
    hbm, peak_kind = peaks()
    achieved = hop_bytes / (hop_ms * 1e-3) / 1e9
    traffic = profile_traffic(f"hop_h12_half_nrhs{NRHS}_{'x'.join(map(str, SHAPE))}")
    # The dominant kernel of the timed solve is the fused CG hop (the fourth hop of an iteration,
    # with x_s += alpha p, r_s -= alpha A p and |r_s|^2 in its epilogue): the largest share of the
    # ncu launch list of a CG iteration.  Timed the same way; it rewrites the slots' x_s and r_s,
    # and this engine solves nothing after it.
    eng.time_hop(reps=3, cg=True)
    cg_ms, cg_bytes = eng.time_hop(reps=20, cg=True)
    cg_achieved = cg_bytes / (cg_ms * 1e-3) / 1e9
    cg_traffic = profile_traffic(f"hop_cg_h12_half_nrhs{NRHS}_{'x'.join(map(str, SHAPE))}")

    # ---- the drop-in FP64 Dslash (reference layout, apply_D), 1 RHS: GB/s against the same peak
    psi1 = eta[NRHS - 1:NRHS].contiguous()
    dout = torch.empty_like(psi1)
    for _ in range(3):
        ctx.apply("D", gauge, MASS, psi1, out=dout)
    cur0 = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(cur0)
    for _ in range(20):
        ctx.apply("D", gauge, MASS, psi1, out=dout)
    e1.record(cur0)
    e1.synchronize()
    ctx.synchronize()
    d_ms = e0.elapsed_time(e1) / 20
    d_bytes = float(np.prod(SHAPE)) * (4 * 144 + 2 * 192)  # 4 links + in/out spinor per site (FP64)
    dslash = {"kernel": "D = m0 - hop/2, reference layout, FP64, 1 RHS (ref_pair_kernel: two threads per site, "
                        "256-bit spinor accesses, parity-split SoA links)",
              "ms_per_launch": d_ms, "algorithmic_bytes_per_launch": d_bytes,
              "achieved": d_bytes / (d_ms * 1e-3) / 1e9, "unit": "GB/s"}
    dslash["frac"] = dslash["achieved"] / peaks()[0]
    dslash["peak"] = peaks()[0]
    dslash.update(naive_rate(np.prod(SHAPE), 1, 192, 144, d_ms))
    dslash.update(ref_gflops(DIRAC.flops_per_matvec_call(3, int(np.prod(SHAPE))), d_ms, "flops_per_matvec_call"))
    del psi1, dout

    # ---- e2e through the public API from pinned host buffers: a stream of K
    # steps, each = host->device copy of its 16 RHS, ctx.solve, device->host copy
    # of its 16 solutions; the copies of neighbouring steps run on a copy stream
    # while the solver runs (double-buffered), and the timed region (CUDA events
    # on the compute stream, after the copy stream drained) spans all K steps.
    b_host = [b.cpu().pin_memory(), b.cpu().pin_memory()]
    x_host = [torch.empty_like(b_host[0]).pin_memory(), torch.empty_like(b_host[0]).pin_memory()]
    b_dev = [torch.empty_like(b), torch.empty_like(b)]
    cur = torch.cuda.current_stream(dev)
    cps = torch.cuda.Stream(dev)

    def e2e_stream(K):
        ev_in = [torch.cuda.Event(), torch.cuda.Event()]
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        e0.record(cur)
        cps.wait_event(e0)
        with torch.cuda.stream(cps):
            b_dev[0].copy_(b_host[0], non_blocking=True)
            ev_in[0].record(cps)
        last = None
        for i in range(K):
            cur.wait_event(ev_in[i % 2])
            if i + 1 < K:
                with torch.cuda.stream(cps):
                    b_dev[(i + 1) % 2].copy_(b_host[(i + 1) % 2], non_blocking=True)
                    ev_in[(i + 1) % 2].record(cps)
            xd, st = ctx.solve(gauge, b_dev[i % 2], MASS, op="eo_normal", tol=TOL, maxiter=4000, inner="half")
            done = torch.cuda.Event()
            done.record(cur)
            cps.wait_event(done)
            with torch.cuda.stream(cps):
                x_host[i % 2].copy_(xd, non_blocking=True)
                xd.record_stream(cps)
            last = st
        drained = torch.cuda.Event()
        drained.record(cps)
        cur.wait_event(drained)
        e1.record(cur)
        e1.synchronize()
        return e0.elapsed_time(e1) / 1e3, last

    e2e_stream(2)  # warm-up
    K = max(3, args.steps)
    t_all, st = e2e_stream(K)
    _, e2e_value = aggregate_over_ranks(t_all / K, NRHS, dist, dev)
    nbytes = b_host[0].numel() * b_host[0].element_size()
    e2e = {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": int(nbytes),
           "d2h_bytes_per_step": int(nbytes), "steps": K,
           "note": "copies of neighbouring steps overlap the solve (copy stream, double buffers)",
           "all_converged": all(s["status"] == 2 for s in st)}
    del b_dev, b_host, x_host

    # ---- serving: Poisson stream of propagator requests, continuous batching
    serve = None
    if args.serve_seconds > 0:
        eng.close()
        serve = run_serving(args, dev)

    # ---- HMC (config C4 couplings on 16^3x32): seconds per trajectory and CG iterations
    hmc = run_hmc_leg(args) if args.hmc_traj > 0 else None

    # ---- CPU baseline (rank 0, N=1): C restatement of the reference's FP64 CG
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(U.cpu().numpy(), b[NRHS - 1].cpu().numpy(), int(np.mean(it64)), args.cpu_seconds)

    if rank == 0:
        line = {
            "metric": METRIC,
            "value": value,
            "unit": "solves/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": t_max * 1e3,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": ("f32 arithmetic on f16 storage" if args.inner == "half" else "f32" if args.inner == "single"
                      else "f64") + " + f64 reliable updates",
            "data": "synthetic (seeded links exp(i*0.2*H), point + Gaussian sources)",
            "config": {"workload": WORKLOAD, "lattice": "x".join(map(str, SHAPE)), "kappa": KAPPA,
                       "nrhs": NRHS, "tol": TOL, "parallelism": f"replicas x{world} (independent solves)",
                       "l2": "working set > 126 MB L2 (no flush needed)"},
            "roofline": {"bound": "hbm",
                         "kernel": "fused CG hop: M^dag y with x_s += alpha p, r_s -= alpha Ap, |r_s|^2 (FP16 storage, "
                                   "12-real links, 16 RHS, EO parity); the largest share of a CG iteration",
                         "achieved": cg_achieved, "peak": hbm, "unit": "GB/s", "frac": cg_achieved / hbm,
                         "peak_kind": peak_kind, "algorithmic_bytes_per_launch": cg_bytes,
                         "bytes_per_site": "8 links x 24 B + 16 RHS x 7 records x 52 B (gathered source; y, p, "
                                           "x_s, r_s read; x_s, r_s written)",
                         "ms_per_launch": cg_ms, "traffic": cg_traffic,
                         **ref_gflops(DIRAC.flops_per_site_dslash(3) * int(np.prod(SHAPE)) // 2 * NRHS, cg_ms,
                                      "flops_per_site_dslash x Vh x 16 RHS (stencil only)")},
            "roofline_plain_hop": {"bound": "hbm", "kernel": "hop K_oe p (FP16 storage, 12-real links, 16 RHS, "
                                                             "EO parity), no epilogue fields",
                                   "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                                   "peak_kind": peak_kind, "algorithmic_bytes_per_launch": hop_bytes,
                                   "ms_per_launch": hop_ms, "traffic": traffic,
                                   **naive_rate(np.prod(SHAPE) // 2, NRHS, 52, 24, hop_ms),
                                   **ref_gflops(DIRAC.flops_per_site_dslash(3) * int(np.prod(SHAPE)) // 2 * NRHS,
                                                hop_ms, "flops_per_site_dslash x Vh x 16 RHS")},
            "gpu_launches": int(launches),
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
            "e2e": e2e,
            "serve": serve,
            "hmc": hmc,
            # kept last, so that a tail of the line still holds them
            "dslash": dslash_native,
            "dslash_fp64_reference_layout": dslash,
            "kappa_0130": light,
            "solve": {"inner": args.inner, "delta": args.delta, "iters_min": min(iters), "iters_max": max(iters),
                      "max_true_res": res, "all_converged": conv,
                      "reliable_updates_max": max(s["reliable_updates"] for s in all_stats[-1])},
            "fp64_cg": {"solves_per_s": fp64_sps * world, "iters": it64, "note": "plain FP64 CG, one RHS at a time"},
            "speedup_vs_fp64": value / (fp64_sps * world),
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def run_hmc_leg(args):
    """Nf=2 HMC with the C4 couplings (16^3x32, beta 5.6, kappa 0.150, MinNorm2 nmd 10, tau 1,
    start exp(i 0.1 H), FP32 force solves at 1e-8 with FP64 reliable updates, FP64 Hamiltonian
    solves at 1e-10) through the drop-in theory and HMC driver: one untimed trajectory, then
    `--hmc-traj` timed ones (wall clock around each, synchronised).  From this start every
    trajectory is rejected (dH ~ 900), which does not change its cost."""
    import contextlib
    import io

    from jaxqft_b200 import hmc_run

    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):  # keep bench's stdout to its one JSON line
        summ = hmc_run.main(["--shape", "16,16,16,32", "--ntraj", str(args.hmc_traj + 1), "--precision", "single"])
    recs = [json.loads(l) for l in buf.getvalue().splitlines() if l.startswith('{"traj"')][1:]
    secs = [r["seconds"] for r in recs]
    iters = [r["cg_iters_total"] for r in recs]
    return {"workload": "C4 HMC trajectory, 16x16x16x32, beta 5.6, kappa 0.150, MinNorm2 nmd 10 tau 1, "
                        "FP32 force solves (FP64 reliable updates) at 1e-8, FP64 Hamiltonian",
            "trajectories": len(recs), "s_per_traj": float(np.mean(secs)),
            "solves_per_traj": float(np.mean([r["solves"] for r in recs])),
            "cg_iters_per_traj": float(np.mean(iters)),
            "us_per_cg_iter": float(np.sum(secs) / max(1, np.sum(iters)) * 1e6),
            "acceptance": summ["acceptance"]}


SERVE_VOLUMES = [(8, 8, 8, 8), (12, 12, 12, 24), (16, 16, 16, 32), (24, 24, 24, 48)]


def run_serving(args, dev):
    """Serving workload: Poisson arrivals over `serve_seconds` at the configured
    mean rate (50/s), volume uniform over {8^4, 12^3x24, 16^3x32, 24^3x48}, kappa
    uniform in [0.120, 0.135], 1-12 point or Gaussian RHS each, on 4 resident
    gauge fields per volume (exp(i*0.2*H), seeds 0-3), admission by HBM budget,
    true residual 1e-10; then the same for `serve_seconds2` at `serve_rate2`, a
    rate one B200 sustains (queue empty when arrivals stop).  Latency includes
    queueing (arrival to last RHS converged); the queue length is sampled."""
    from jaxqft_b200.serving import PropagatorServer, serve_once, warm_server

    server = PropagatorServer(SERVE_VOLUMES, gauge_seeds=(0, 1, 2, 3), nslots=16, inner="half", tol=TOL,
                              device=dev, keep_solutions=False)
    warm_server(server)  # every engine allocated, tuned and graph-captured before the timed streams
    out = serve_once(server, args.serve_rate, args.serve_seconds)
    out.update({"volumes": ["x".join(map(str, v)) for v in SERVE_VOLUMES], "gauge_fields_per_volume": 4,
                "hbm_budget_GB": server.hbm_budget / 1e9, "peak_engine_GB": server.peak_engine_bytes / 1e9})
    if args.serve_seconds2 > 0:
        out["sustained"] = serve_once(server, args.serve_rate2, args.serve_seconds2, seed=2)
        out["sustained"].pop("per_volume", None)
    server.close()
    return out


# --------------------------------------------------------------------------- CPU legs
# Both CPU legs (the cpu_baseline of our arm and the --impl reference arm) time the
# same unit: one call of the C restatement's FP64 CG running CPU_ITERS_PER_CALL
# iterations of M^dag M on the full 24^3x48 system (a quarter of a solve, so
# per-call set-up is amortised the same way in both), converted to solves/s with
# the iteration count plain FP64 CG needs to reach 1e-10 on this system.
CPU_ITERS_PER_CALL = 39


def cpu_seconds_per_iter(cw, be, calls: int):
    """Per-iteration seconds of `calls` timed CG calls (x = 0 start, no early stop)."""
    out = []
    for _ in range(calls):
        t0 = time.perf_counter()
        cw.cg(be, 0.0, CPU_ITERS_PER_CALL)
        out.append((time.perf_counter() - t0) / CPU_ITERS_PER_CALL)
    return out


def cpu_baseline(U4, b_full, iters_to_converge: int, seconds: float):
    """The C restatement on all host cores for about `seconds` (whole calls)."""
    from oracle import cpu as C
    from oracle import wilson as W

    C.build()
    cw = C.CpuWilson(U4, SHAPE, BC, MASS)
    be = W.pack(b_full[None], 0)[0]
    first = cpu_seconds_per_iter(cw, be, 1)[0]  # warm-up call (thread start, first touch)
    calls = max(1, int(seconds / max(first * CPU_ITERS_PER_CALL, 1e-6)))
    per = float(np.mean(cpu_seconds_per_iter(cw, be, calls)))
    return {"value": 1.0 / (per * iters_to_converge), "unit": "solves/s", "cores": C.threads(), "kind": "port",
            "sample": f"{calls} calls x {CPU_ITERS_PER_CALL} FP64 CG iterations of M^dag M on the full 24^3x48 "
                      f"system, 1 RHS; solves/s = 1/(s/iter x {iters_to_converge} iters to 1e-10)",
            "s_per_iter": per}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    # The reference (JAX) is not installable offline here; its CPU path is timed
    # through the C restatement of its even-odd CG (oracle/c) on all host cores.
    import torch

    from oracle import cpu as C
    from oracle import wilson as W

    U, eta = make_inputs(torch, torch.device("cpu"), seed=0)
    C.build()
    cw = C.CpuWilson(U.numpy(), SHAPE, BC, MASS)
    be = cw.normal(W.pack(eta[12:13].numpy(), 0)[0])  # an even RHS of the system; only timing is used
    cpu_seconds_per_iter(cw, be, args.warmup)
    per = float(np.mean(cpu_seconds_per_iter(cw, be, args.steps)))
    iters = args.ref_iters
    value = 1.0 / (per * iters)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": per * CPU_ITERS_PER_CALL * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "lattice": "x".join(map(str, SHAPE)), "kappa": KAPPA},
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": C.threads(), "kind": "port",
                             "sample": f"{CPU_ITERS_PER_CALL} FP64 CG iterations per step on the full system, 1 RHS; "
                                       f"solves/s = 1/(s/iter x {iters} iterations FP64 CG needs to 1e-10)"},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "jaxQFT needs JAX, which is not installable offline; its EO CG is timed via the C restatement"}
    print(json.dumps(line), flush=True)


def run_profile_dslash(args):
    """Profiling driver for the FP64 Dslash, 1 RHS: the drop-in D on the reference
    layout (3 warm-up applications, then `--profile-dslash` applications between
    cudaProfilerStart/Stop), or with --dslash-layout internal the EO hop of the
    FP64 engine (one more launch inside the range)."""
    import torch

    from jaxqft_b200 import lib as L

    global SHAPE
    SHAPE = tuple(int(v) for v in args.shape.split(","))
    dev = torch.device("cuda", 0)
    ctx = L.WilsonContext(SHAPE, bc=BC, device=dev)
    U, eta = make_inputs(torch, dev, seed=0)
    gauge = ctx.gauge(U)
    if args.dslash_layout == "update":  # the FP64 hop of the reliable update of the 16-slot FP16 engine
        del U, eta
        eng = L.Engine(ctx, gauge, NRHS, op="eo_normal", inner="half", tol=TOL, maxiter=10)
        eng.time_hop(reps=3, update=True)
        torch.cuda.synchronize()
        torch.cuda.cudart().cudaProfilerStart()
        ms, byts = eng.time_hop(reps=args.profile_dslash, update=True)
        torch.cuda.cudart().cudaProfilerStop()
        eng.close()
        print(json.dumps({"profile": f"FP64 reliable-update hop, {NRHS} RHS in lanes", "shape": SHAPE, "ms": ms,
                          "GBps": byts / ms / 1e6}), flush=True)
        return
    if args.dslash_layout == "internal":  # the EO hop of the FP64 1-RHS engine (SoA fields, 18-real links)
        del U, eta
        eng = L.Engine(ctx, gauge, 1, op="eo_normal", inner="double", tol=TOL, maxiter=10)
        eng.time_hop(reps=3)
        torch.cuda.synchronize()
        torch.cuda.cudart().cudaProfilerStart()
        ms, byts = eng.time_hop(reps=args.profile_dslash)
        torch.cuda.cudart().cudaProfilerStop()
        eng.close()
        print(json.dumps({"profile": "FP64 EO hop, internal layout, 1 RHS", "shape": SHAPE, "ms": ms,
                          "GBps": byts / ms / 1e6}), flush=True)
        return
    psi = eta[NRHS - 1:NRHS].contiguous()
    del U, eta
    out = torch.empty_like(psi)
    for _ in range(3):
        ctx.apply("D", gauge, MASS, psi, out=out)
    ctx.synchronize()
    torch.cuda.cudart().cudaProfilerStart()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.profile_dslash):
        ctx.apply("D", gauge, MASS, psi, out=out)
    e1.record()
    e1.synchronize()
    torch.cuda.cudart().cudaProfilerStop()
    ctx.synchronize()
    ms = e0.elapsed_time(e1) / args.profile_dslash
    byts = float(np.prod(SHAPE)) * 960.0
    print(json.dumps({"profile": "FP64 D, reference layout, 1 RHS", "shape": SHAPE, "ms": ms,
                      "GBps": byts / ms / 1e6}), flush=True)


def run_profile(args):
    """Profiling driver: a fixed number of batched CG iterations of the same
    solver, bracketed by cudaProfilerStart/Stop so that
    `ncu --profile-from-start off` captures only those launches."""
    import torch

    from jaxqft_b200 import lib as L

    global SHAPE
    SHAPE = tuple(int(v) for v in args.shape.split(","))
    dev = torch.device("cuda", 0)
    ctx = L.WilsonContext(SHAPE, bc=BC, device=dev)
    U, eta = make_inputs(torch, dev, seed=0)
    gauge = ctx.gauge(U)
    del U
    b = ctx.apply("SCHUR_E_DAG", gauge, MASS, eta[:args.nrhs] * even_mask(torch, dev), normalized=True)
    del eta
    eng = L.Engine(ctx, gauge, args.nrhs, op="eo_normal", inner=args.inner, tol=1e-14, maxiter=100000,
                   use_graph=not args.no_graph)
    eng.admit(np.arange(args.nrhs), b, MASS)
    eng.step(3)
    eng.poll()
    torch.cuda.synchronize()
    torch.cuda.cudart().cudaProfilerStart()
    t0 = time.perf_counter()
    eng.step(args.profile_iters)
    eng.poll()
    t1 = time.perf_counter()
    torch.cuda.cudart().cudaProfilerStop()
    ms, by = eng.time_hop(reps=10)
    print(json.dumps({"profile": "eo_normal CG iterations", "shape": SHAPE, "nrhs": args.nrhs, "inner": args.inner,
                      "iters": args.profile_iters, "ms_per_iter_wall": (t1 - t0) * 1e3 / args.profile_iters,
                      "hop_us": ms * 1e3, "hop_GBps": by / ms / 1e6}), flush=True)


def ref_gflops(flops, ms, how):
    """GFLOP/s on the reference's own flop count (jaxqft/fermions/wilson.py:349-437)."""
    return {"ref_flops_per_launch": int(flops), "ref_gflops": float(flops) / (ms * 1e-3) / 1e9,
            "ref_flops_count": f"WilsonDiracOperator.{how} (nc=3, sparse gamma)"}


def naive_rate(sites, nrhs, spinor_bytes, link_bytes, ms):
    """The lattice-QCD "naive" bandwidth convention, reported beside the
    algorithmic figure: per target site and RHS, 8 neighbour spinors read and one
    written (9 S), plus 8 links per target site, with no credit for cache reuse.
    It over-counts DRAM traffic, so it is never the roofline numerator."""
    b = float(sites) * (nrhs * 9 * spinor_bytes + 8 * link_bytes)
    return {"naive_bytes_per_launch": b, "naive_gbs": b / (ms * 1e-3) / 1e9,
            "naive_convention": "9S+8L per target site (S, L: stored spinor and link bytes), no cache reuse"}


def main():
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--delta", type=float, default=0.1, help="reliable-update threshold of the mixed solver")
    ap.add_argument("--serve-seconds", type=float, default=4.0, help="serving leg: seconds of Poisson arrivals (0: off)")
    ap.add_argument("--serve-rate", type=float, default=50.0, help="serving leg: mean requests per second")
    ap.add_argument("--serve-seconds2", type=float, default=10.0,
                    help="serving leg: seconds of arrivals at --serve-rate2 (0: off)")
    ap.add_argument("--serve-rate2", type=float, default=12.0,
                    help="serving leg: a mean rate one B200 sustains without queue growth")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--hmc-traj", type=int, default=2, help="HMC leg: timed C4 trajectories on 16^3x32 (0: off)")
    ap.add_argument("--fp64-all", action="store_true", help="time plain FP64 CG on all 16 RHS (default 4)")
    ap.add_argument("--profile-iters", type=int, default=0,
                    help="profiling driver: run this many CG iterations between cudaProfilerStart/Stop")
    ap.add_argument("--shape", default="24,24,24,48", help="lattice for --profile-iters")
    ap.add_argument("--nrhs", type=int, default=NRHS, help="RHS count for --profile-iters")
    ap.add_argument("--inner", default="half", help="iterated precision for --profile-iters")
    ap.add_argument("--no-graph", action="store_true",
                    help="--profile-iters: launch kernels directly (ncu cannot profile kernels inside graphs "
                         "with conditional nodes)")
    ap.add_argument("--ref-iters", type=int, default=153,
                    help="FP64 CG iterations to 1e-10 on this system: plain FP64 CG needs 152-154 on each of the "
                         "16 RHS (measured with --fp64-all)")
    ap.add_argument("--profile-dslash", type=int, default=0,
                    help="profiling driver: this many FP64 Dslash applications (on --shape)")
    ap.add_argument("--dslash-layout", default="reference", choices=["reference", "internal", "update"],
                    help="--profile-dslash: reference-layout D, the internal-layout EO hop, or the FP64 "
                         "reliable-update hop of the 16-slot engine")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.profile_dslash > 0:
        run_profile_dslash(args)
    elif args.profile_iters > 0:
        run_profile(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
