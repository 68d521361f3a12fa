"""The hot path under the index-checking build (libwilson_sm100_check.so).

compute-sanitizer is not available to this project, so out-of-range accesses
are looked for by a build of the same sources with WL_BOUNDS_CHECK=1: every
compact site index that a kernel decodes, sweeps or gathers is compared with
the half volume; a bad one is counted, and site 0 is used in its place (no
assert, no trap), and wl_bounds_errors() returns the count.  A fresh process
loads that library and runs every kernel family at small sizes, on an even
cubic lattice and on an anisotropic one with a complex boundary phase: the
drop-in D (row-staged TMA kernel), the Schur normal operator, a batched FP16
solve (RHS-in-lanes hops, FP64 tiled update hops), FP64 and FP32 solves, the
pseudofermion force and the gauge kernels.  It must report zero bad indices,
and the checked build must still agree with the oracle (D at 1e-13, every
solve at an FP64 true residual <= 1e-10).
"""

import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("CUDA device required", allow_module_level=True)

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import ctypes, json, os, sys
import numpy as np, torch
sys.path.insert(0, ROOT)
from jaxqft_b200 import build as B, lib as L
from oracle import wilson as W

if not os.path.exists(L.CHECK_LIB_PATH):  # build() makes it beside the release library
    B.build_check()
lib = L.load_library(L.CHECK_LIB_PATH)
rep = {"library": lib._name, "cases": []}
for shape, bc in (((4, 4, 4, 8), (1, 1, 1, -1)), ((2, 4, 6, 4), (1, 1, 1j, -1))):
    rng = np.random.default_rng(3)
    U = W.hot_links(rng, shape, 1, 0.3)
    m = W.kappa_to_mass(0.12)
    ctx = L.WilsonContext(shape, bc=bc)
    g = ctx.gauge(torch.from_numpy(U[0]))
    psi = W.gaussian_spinor(rng, shape, 8)
    d = ctx.apply("D", g, m, torch.from_numpy(psi)).cpu().numpy()
    ref = W.apply_D(U, psi[:2], m, bc)
    err_d = max(float(np.linalg.norm(d[r] - ref[r]) / np.linalg.norm(ref[r])) for r in range(2))
    b = W.project(psi, 0)
    ctx.apply("SCHUR_E_NORMAL", g, m, torch.from_numpy(b), normalized=True)
    stats = []
    for rhs, op, inner in ((b, "eo_normal", "half"), (b[:1], "eo_normal", "double"), (psi[:2], "normal", "single")):
        _, st = ctx.solve(g, torch.from_numpy(rhs), m, op=op, tol=1e-10, maxiter=3000, inner=inner)
        stats += [(s["status"], s["true_res"]) for s in st]
    ctx.pf_force(g, torch.from_numpy(psi[0]), torch.from_numpy(psi[1]))
    Ut = torch.from_numpy(U)
    F = ctx.gauge_force(Ut, 5.6)
    ctx.gauge_evolve(0.05, F, Ut)
    ctx.plaquette_sum(Ut)
    torch.cuda.synchronize()
    first = ctypes.c_longlong(0)
    n = int(lib.wl_bounds_errors(ctypes.byref(first)))
    rep["cases"].append({"shape": list(shape), "bad_indices": n, "first_bad": int(first.value), "err_D": err_d,
                         "solves": stats})
print(json.dumps(rep))
"""


def test_hot_path_has_no_out_of_range_site_index():
    res = subprocess.run([sys.executable, "-c", CHILD.replace("ROOT", repr(ROOT), 1)], cwd=ROOT,
                         capture_output=True, text=True, timeout=900)
    assert res.returncode == 0, res.stdout[-2000:] + res.stderr[-4000:]
    rep = json.loads(res.stdout.strip().splitlines()[-1])
    assert rep["library"].endswith("libwilson_sm100_check.so"), rep["library"]
    for case in rep["cases"]:
        assert case["bad_indices"] == 0, case
        assert case["err_D"] < 1e-13, case
        assert len(case["solves"]) == 8 + 1 + 2
        for status, true_res in case["solves"]:
            assert status == 2 and true_res <= 1e-10, case
