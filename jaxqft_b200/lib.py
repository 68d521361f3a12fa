"""ctypes binding of libwilson_sm100.so (the C-ABI in include/wilson_sm100.h).

There is no CPU fallback: every compute entry point requires the in-tree CUDA
library and a CUDA device, and raises ``RuntimeError`` otherwise.  Field
arguments are torch CUDA tensors (complex128, contiguous) whose device
pointers are handed to the library; ownership stays with the caller.
"""

from __future__ import annotations

import ctypes
import os
from typing import Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libwilson_sm100.so")
# the same library compiled with device-side index checks (WL_BOUNDS_CHECK)
CHECK_LIB_PATH = os.path.join(HERE, "libwilson_sm100_check.so")
HEADER_PATH = os.path.join(os.path.dirname(HERE), "include", "wilson_sm100.h")

# status codes (wl_status)
WL_OK, WL_ERR_ARG, WL_ERR_OOM, WL_NOT_CONVERGED, WL_ERR_NAN, WL_ERR_TIMEOUT, WL_ERR_CUDA, WL_ERR_STATE = range(8)
STATUS_NAMES = {
    WL_OK: "OK", WL_ERR_ARG: "ERR_ARG", WL_ERR_OOM: "ERR_OOM", WL_NOT_CONVERGED: "NOT_CONVERGED",
    WL_ERR_NAN: "ERR_NAN", WL_ERR_TIMEOUT: "ERR_TIMEOUT", WL_ERR_CUDA: "ERR_CUDA", WL_ERR_STATE: "ERR_STATE",
}
PREC = {"double": 0, "single": 1, "half": 2, "fp64": 0, "fp32": 1, "fp16": 2}
OPS = dict(D=0, DDAG=1, DDAGD=2, HOP=3, HOP_DAG=4, K_OE=5, K_EO=6, KDAG_OE=7, KDAG_EO=8,
           SCHUR_E=9, SCHUR_E_DAG=10, SCHUR_O=11, SCHUR_E_NORMAL=12)
FLAG_NORMALIZED = 1
SOLVE_NORMAL, SOLVE_EO_NORMAL = 0, 1
# per-RHS solver status (wl_solve_stats.status)
SLOT_CONVERGED, SLOT_MAXITER, SLOT_BREAKDOWN, SLOT_NAN = 2, 3, 4, 5

# Every symbol the header declares (checked by tests/test_abi.py).
EXPORTS = (
    "wl_version", "wl_ctx_create", "wl_ctx_destroy", "wl_last_error", "wl_ctx_set_stream",
    "wl_ctx_synchronize", "wl_eo_maps", "wl_gauge_create", "wl_gauge_update", "wl_gauge_unitarity",
    "wl_gauge_destroy", "wl_apply", "wl_solve", "wl_engine_create", "wl_engine_destroy", "wl_engine_admit",
    "wl_engine_step", "wl_engine_run", "wl_engine_poll", "wl_engine_poll_async", "wl_engine_poll_ready", "wl_engine_retire", "wl_engine_bytes", "wl_pf_force",
    "wl_engine_stream", "wl_engine_time_hop", "wl_engine_time_update_hop", "wl_engine_time_cg_hop", "wl_kernel_launches", "wl_engine_debug_apply",
    "wl_apply_schur_normal_noalloc", "wl_gauge_force", "wl_gauge_evolve", "wl_gauge_plaquette_sum",
    "wl_momentum_kinetic", "wl_pion_correlator", "wl_bounds_errors", "wl_random_spinor", "wl_random_algebra",
    "wl_field_dots", "wl_field_combine",
)


class WLGeometry(ctypes.Structure):
    _fields_ = [("dims", ctypes.c_int * 4), ("bc_re", ctypes.c_double * 4), ("bc_im", ctypes.c_double * 4)]


class WLSolveParams(ctypes.Structure):
    _fields_ = [
        ("op", ctypes.c_int), ("inner_prec", ctypes.c_int), ("tol", ctypes.c_double), ("maxiter", ctypes.c_int),
        ("delta", ctypes.c_double), ("use_x0", ctypes.c_int), ("use_graph", ctypes.c_int),
        ("check_every", ctypes.c_int),
    ]


class WLSolveStats(ctypes.Structure):
    _fields_ = [("iters", ctypes.c_int), ("reliable_updates", ctypes.c_int), ("status", ctypes.c_int),
                ("true_res", ctypes.c_double)]


_lib = None


def load_library(path: Optional[str] = None) -> ctypes.CDLL:
    """Load (and declare prototypes of) the in-tree CUDA library.  Builds it
    with nvcc first if it is missing and a toolkit is present."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or LIB_PATH
    if not os.path.exists(path):
        from . import build as _build

        _build.build()
    if not os.path.exists(path):
        raise RuntimeError(f"libwilson_sm100.so not found at {path}; run python -m jaxqft_b200.build")
    lib = ctypes.CDLL(path)
    vp, i, d, u = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_uint
    pi, pd = ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)
    sig = {
        "wl_version": (i, []),
        "wl_ctx_create": (i, [ctypes.POINTER(WLGeometry), i, ctypes.POINTER(vp)]),
        "wl_ctx_destroy": (None, [vp]),
        "wl_last_error": (ctypes.c_char_p, [vp]),
        "wl_ctx_set_stream": (i, [vp, vp]),
        "wl_ctx_synchronize": (i, [vp]),
        "wl_eo_maps": (i, [vp, vp, vp, vp]),
        "wl_gauge_create": (i, [vp, vp, ctypes.POINTER(vp)]),
        "wl_gauge_update": (i, [vp, vp]),
        "wl_gauge_unitarity": (i, [vp, pd]),
        "wl_gauge_destroy": (None, [vp]),
        "wl_apply": (i, [vp, vp, i, d, u, vp, vp, i]),
        "wl_solve": (i, [vp, vp, ctypes.POINTER(WLSolveParams), pd, vp, vp, i, ctypes.POINTER(WLSolveStats)]),
        "wl_engine_create": (i, [vp, vp, ctypes.POINTER(WLSolveParams), i, ctypes.POINTER(vp)]),
        "wl_engine_destroy": (None, [vp]),
        "wl_engine_admit": (i, [vp, pi, i, vp, pd, pd, pi]),
        "wl_engine_step": (i, [vp, i]),
        "wl_engine_run": (i, [vp, i]),
        "wl_engine_poll": (i, [vp, pi, pi]),
        "wl_engine_poll_async": (i, [vp]),
        "wl_engine_poll_ready": (i, [vp, pi, pi]),
        "wl_engine_retire": (i, [vp, i, vp, ctypes.POINTER(WLSolveStats)]),
        "wl_engine_bytes": (ctypes.c_int64, [vp, i, i, i]),
        "wl_pf_force": (i, [vp, vp, vp, vp, d, i, vp]),
        "wl_engine_stream": (vp, [vp]),
        "wl_engine_time_hop": (i, [vp, i, pd, pd]),
        "wl_engine_time_update_hop": (i, [vp, i, pd, pd]),
        "wl_engine_time_cg_hop": (i, [vp, i, pd, pd]),
        "wl_kernel_launches": (ctypes.c_int64, []),
        "wl_bounds_errors": (ctypes.c_int64, [ctypes.POINTER(ctypes.c_longlong)]),
        "wl_engine_debug_apply": (i, [vp, i, d, vp, vp]),
        "wl_apply_schur_normal_noalloc": (i, [vp, vp, d, u, vp, vp, i]),
        "wl_gauge_force": (i, [vp, vp, i, d, vp]),
        "wl_gauge_evolve": (i, [vp, vp, vp, i, d, vp]),
        "wl_gauge_plaquette_sum": (i, [vp, vp, i, pd]),
        "wl_momentum_kinetic": (i, [vp, vp, i, pd]),
        "wl_pion_correlator": (i, [vp, vp, i, i, pd]),
        "wl_random_spinor": (i, [vp, ctypes.c_uint64, ctypes.c_uint64, i, vp]),
        "wl_field_dots": (i, [vp, i, ctypes.POINTER(vp), ctypes.POINTER(vp), ctypes.c_int64, pd]),
        "wl_field_combine": (i, [vp, i, ctypes.POINTER(vp), pd, ctypes.c_int64, vp]),
        "wl_random_algebra": (i, [vp, ctypes.c_uint64, ctypes.c_uint64, i, d, vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class WilsonError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


def kernel_launches() -> int:
    """Kernels launched by libwilson_sm100 in this process so far."""
    return int(load_library().wl_kernel_launches())


def _require_cuda():
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("the B200 Wilson-fermion path requires a CUDA device (no CPU fallback)")
    return torch


def _ptr(t) -> int:
    return int(t.data_ptr())


def _c128(t, device):
    import torch

    if isinstance(t, np.ndarray):
        t = torch.from_numpy(np.ascontiguousarray(t))
    if t.dtype != torch.complex128:
        t = t.to(torch.complex128)
    if t.device != device:
        t = t.to(device)
    return t.contiguous()


class Gauge:
    """Device copies of one gauge configuration (internal parity-split FP64 /
    FP32 / FP16 layouts built by the library)."""

    def __init__(self, ctx: "WilsonContext", U):
        self.ctx = ctx
        lib = ctx.lib
        U = _c128(U, ctx.device)
        h = ctypes.c_void_p()
        ctx._check(lib.wl_gauge_create(ctx.handle, _ptr(U), ctypes.byref(h)))
        self.handle = h
        self._src = U  # keep the source alive until the async copy has run

    def update(self, U):
        U = _c128(U, self.ctx.device)
        self.ctx._check(self.ctx.lib.wl_gauge_update(self.handle, _ptr(U)))
        self._src = U

    def unitarity(self) -> float:
        v = ctypes.c_double()
        self.ctx._check(self.ctx.lib.wl_gauge_unitarity(self.handle, ctypes.byref(v)))
        return float(v.value)

    def close(self):
        if getattr(self, "handle", None) is not None and self.handle.value:
            self.ctx.lib.wl_gauge_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class WilsonContext:
    """One lattice geometry on one CUDA device (wraps wl_ctx)."""

    def __init__(self, lattice_shape: Sequence[int], bc=(1, 1, 1, 1), device=None):
        torch = _require_cuda()
        self.lib = load_library()
        if len(lattice_shape) != 4:
            raise ValueError("the SU(3) Wilson path is 4-dimensional")
        self.lattice_shape = tuple(int(v) for v in lattice_shape)
        if any(v < 2 or v % 2 for v in self.lattice_shape):
            raise ValueError("every lattice extent must be even and >= 2 (even/odd layout)")
        self.device = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        self.volume = int(np.prod(self.lattice_shape))
        g = WLGeometry()
        for mu in range(4):
            g.dims[mu] = self.lattice_shape[mu]
            p = complex(bc[mu])
            g.bc_re[mu] = p.real
            g.bc_im[mu] = p.imag
        h = ctypes.c_void_p()
        rc = self.lib.wl_ctx_create(ctypes.byref(g), int(self.device.index or 0), ctypes.byref(h))
        if rc != WL_OK:
            raise WilsonError(rc, self.lib.wl_last_error(None).decode())
        self.handle = h
        self.bc = tuple(complex(b) for b in bc)
        self.set_stream(torch.cuda.current_stream(self.device))

    def set_stream(self, stream):
        self._check(self.lib.wl_ctx_set_stream(self.handle, ctypes.c_void_p(int(stream.cuda_stream))))

    def _check(self, rc: int):
        if rc != WL_OK:
            raise WilsonError(rc, self.lib.wl_last_error(self.handle).decode())

    def gauge(self, U) -> Gauge:
        return Gauge(self, U)

    def synchronize(self):
        self._check(self.lib.wl_ctx_synchronize(self.handle))

    # ------------------------------------------------------------ operators
    def apply(self, op: str, gauge: Gauge, mass: float, psi, normalized: bool = False, out=None):
        """out = op(psi) for psi of shape (nrhs, Lx, Ly, Lz, Lt, 4, 3) or (Lx..Lt, 4, 3)."""
        import torch

        psi = _c128(psi, self.device)
        nrhs = psi.numel() // (12 * self.volume)
        if nrhs * 12 * self.volume != psi.numel():
            raise ValueError(f"field of {psi.numel()} elements does not match lattice {self.lattice_shape}")
        if out is None:
            out = torch.empty_like(psi)
        if nrhs == 0:  # an empty batch maps to an empty result, as the reference's vmapped operators do
            return out
        flags = FLAG_NORMALIZED if normalized else 0
        self._check(self.lib.wl_apply(self.handle, gauge.handle, OPS[op], float(mass), flags, _ptr(psi), _ptr(out),
                                      nrhs))
        return out

    def pf_force(self, gauge: Gauge, X, Y, coef: float = 1.0, F=None):
        """F (+)= coef * pseudofermion_force_from_solution(U, X, Y) for one configuration."""
        import torch

        X = _c128(X, self.device)
        Y = _c128(Y, self.device)
        acc = F is not None
        if F is None:
            F = torch.empty((4, *self.lattice_shape, 3, 3), dtype=torch.complex128, device=self.device)
        self._check(self.lib.wl_pf_force(self.handle, gauge.handle, _ptr(X), _ptr(Y), float(coef), int(acc),
                                         _ptr(F)))
        return F

    # ------------------------------------------------------------ gauge sector
    def _links(self, x, name):
        """Reference-layout BMXYIJ complex128 batch [B, 4, *L, 3, 3] on this device."""
        x = _c128(x, self.device)
        if x.numel() % (36 * self.volume) != 0:
            raise ValueError(f"{name} of {x.numel()} elements does not match [B, 4, {self.lattice_shape}, 3, 3]")
        return x, x.numel() // (36 * self.volume)

    def gauge_force(self, U, beta: float, out=None):
        """-(beta/3) TA(U_mu V_mu^dag) per link (su3_ym.py force), U of shape [B, 4, *L, 3, 3]."""
        import torch

        U, B = self._links(U, "U")
        if out is None:
            out = torch.empty_like(U)
        self._check(self.lib.wl_gauge_force(self.handle, _ptr(U), B, float(beta), _ptr(out)))
        return out

    def gauge_evolve(self, dt: float, P, U, out=None):
        """exp(dt P) U per link (su3_ym.py evolve_q with exp_method "expm")."""
        import torch

        U, B = self._links(U, "U")
        P, BP = self._links(P, "P")
        if BP != B:
            raise ValueError("P and U batch sizes differ")
        if out is None:
            out = torch.empty_like(U)
        self._check(self.lib.wl_gauge_evolve(self.handle, _ptr(P), _ptr(U), B, float(dt), _ptr(out)))
        return out

    def plaquette_sum(self, U) -> np.ndarray:
        """sum_{x, mu<nu} Re Tr U_p per configuration (FP64, host array)."""
        U, B = self._links(U, "U")
        out = np.zeros(B, dtype=np.float64)
        self._check(self.lib.wl_gauge_plaquette_sum(self.handle, _ptr(U), B,
                                                    out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return out

    def kinetic(self, P) -> np.ndarray:
        """-1/2 sum Re Tr P P per configuration (FP64, host array)."""
        P, B = self._links(P, "P")
        out = np.zeros(B, dtype=np.float64)
        self._check(self.lib.wl_momentum_kinetic(self.handle, _ptr(P), B,
                                                 out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return out

    def field_dots(self, pairs) -> np.ndarray:
        """<a, b> = sum conj(a) b for each (a, b) in `pairs` (complex128 device
        tensors of equal size), in one pass per pair on the device (wl_field_dots)."""
        pairs = [(_c128(a, self.device), _c128(b, self.device)) for a, b in pairs]
        n = len(pairs)
        out = np.zeros(2 * n, dtype=np.float64)
        length = pairs[0][0].numel()
        if any(a.numel() != length or b.numel() != length for a, b in pairs):
            raise ValueError("field_dots: fields of different sizes")
        A = (ctypes.c_void_p * n)(*[_ptr(a) for a, _ in pairs])
        B = (ctypes.c_void_p * n)(*[_ptr(b) for _, b in pairs])
        self._check(self.lib.wl_field_dots(self.handle, n, A, B, int(length),
                                           out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return out[0::2] + 1j * out[1::2]

    def field_combine(self, coefs, xs, out=None):
        """out = sum_k coefs[k] xs[k] (complex coefficients) on the device (wl_field_combine)."""
        import torch

        xs = [_c128(x, self.device) for x in xs]
        n = len(xs)
        c = np.empty(2 * n, dtype=np.float64)
        c[0::2] = np.real(np.asarray(coefs, dtype=np.complex128))
        c[1::2] = np.imag(np.asarray(coefs, dtype=np.complex128))
        if out is None:
            out = torch.empty_like(xs[0])
        X = (ctypes.c_void_p * n)(*[_ptr(x) for x in xs])
        self._check(self.lib.wl_field_combine(self.handle, n, X, c.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                              int(xs[0].numel()), _ptr(out)))
        return out

    def random_spinor(self, n: int, seed: int, stream: int):
        """n complex Gaussian fields [n, *L, 4, 3], E|z|^2 = 1, from the device
        generator (wl_random_spinor); (seed, stream) fixes the field."""
        import torch

        out = torch.empty((int(n), *self.lattice_shape, 4, 3), dtype=torch.complex128, device=self.device)
        self._check(self.lib.wl_random_spinor(self.handle, int(seed) & (2**64 - 1), int(stream) & (2**64 - 1),
                                              int(n), _ptr(out)))
        return out

    def random_algebra(self, batch: int, seed: int, stream: int, scale: float = 1.0):
        """TA(scale (G1 + i G2)) per link, [batch, 4, *L, 3, 3] (BMXYIJ), from the
        device generator (wl_random_algebra)."""
        import torch

        out = torch.empty((int(batch), 4, *self.lattice_shape, 3, 3), dtype=torch.complex128, device=self.device)
        self._check(self.lib.wl_random_algebra(self.handle, int(seed) & (2**64 - 1), int(stream) & (2**64 - 1),
                                               int(batch), float(scale), _ptr(out)))
        return out

    def pion_correlator(self, prop, source_t: int) -> np.ndarray:
        """C(dt), dt = 0..Lt-1, of point-source propagator columns prop [ncol, *L, 4, 3]
        (measurements.py:375-390): sum of |S|^2 over columns, spin, colour and the timeslice."""
        prop = _c128(prop, self.device)
        ncol = prop.numel() // (12 * self.volume)
        if ncol * 12 * self.volume != prop.numel():
            raise ValueError(f"propagator of {prop.numel()} elements does not match lattice {self.lattice_shape}")
        out = np.zeros(self.lattice_shape[3], dtype=np.float64)
        self._check(self.lib.wl_pion_correlator(self.handle, _ptr(prop), ncol, int(source_t),
                                                out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return out

    def eo_maps(self):
        vh = self.volume // 2
        even = np.zeros(vh, dtype=np.int32)
        odd = np.zeros(vh, dtype=np.int32)
        nbr = np.zeros((2, 4, 2, vh), dtype=np.int32)
        self._check(self.lib.wl_eo_maps(self.handle, even.ctypes.data, odd.ctypes.data, nbr.ctypes.data))
        return even, odd, nbr

    # ------------------------------------------------------------ solves
    def solve(self, gauge: Gauge, b, masses, op: str = "eo_normal", tol: float = 1e-10, maxiter: int = 1000,
              inner: str = "double", delta: float = 0.1, x0=None, use_graph: bool = True, check_every: int = 8):
        """Batched CG for nrhs systems sharing `gauge`.  Returns (x, stats list)."""
        import torch

        b = _c128(b, self.device)
        nrhs = b.numel() // (12 * self.volume)
        masses = np.broadcast_to(np.asarray(masses, dtype=np.float64), (nrhs,)).copy()
        if x0 is not None:
            x = _c128(x0, self.device).clone()
        else:
            x = torch.empty_like(b)
        p = WLSolveParams()
        p.op = SOLVE_EO_NORMAL if op == "eo_normal" else SOLVE_NORMAL
        p.inner_prec = PREC[inner]
        p.tol = float(tol)
        p.maxiter = int(maxiter)
        p.delta = float(delta if inner != "double" else 0.0)
        p.use_x0 = int(x0 is not None)
        p.use_graph = int(bool(use_graph))
        p.check_every = int(check_every)
        if nrhs == 0:  # nothing to solve: empty solution, no stats
            return x, []
        stats = (WLSolveStats * nrhs)()
        rc = self.lib.wl_solve(self.handle, gauge.handle, ctypes.byref(p),
                               masses.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), _ptr(b), _ptr(x), nrhs, stats)
        st = [dict(iters=s.iters, reliable_updates=s.reliable_updates, status=s.status, true_res=s.true_res)
              for s in stats]
        if rc not in (WL_OK, WL_NOT_CONVERGED):
            self._check(rc)
        return x, st

    def engine_bytes(self, op: str, inner: str, nslots: int) -> int:
        return int(self.lib.wl_engine_bytes(self.handle, SOLVE_EO_NORMAL if op == "eo_normal" else SOLVE_NORMAL,
                                            PREC[inner], int(nslots)))

    def close(self):
        if getattr(self, "handle", None) is not None and self.handle.value:
            self.lib.wl_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Engine:
    """Continuous-batching CG engine (wl_engine): fixed RHS slots on one gauge."""

    def __init__(self, ctx: WilsonContext, gauge: Gauge, nslots: int, op: str = "eo_normal", inner: str = "half",
                 tol: float = 1e-10, maxiter: int = 2000, delta: float = 0.1, use_graph: bool = True):
        self.ctx, self.gauge, self.nslots = ctx, gauge, int(nslots)
        p = WLSolveParams()
        p.op = SOLVE_EO_NORMAL if op == "eo_normal" else SOLVE_NORMAL
        p.inner_prec = PREC[inner]
        p.tol = float(tol)
        p.maxiter = int(maxiter)
        p.delta = float(delta if inner != "double" else 0.0)
        p.use_graph = int(bool(use_graph))
        p.check_every = 8
        h = ctypes.c_void_p()
        ctx._check(ctx.lib.wl_engine_create(ctx.handle, gauge.handle, ctypes.byref(p), self.nslots, ctypes.byref(h)))
        self.handle = h
        self._inputs = []

    def admit(self, slots, b, masses, tols=None, maxiters=None):
        b = _c128(b, self.ctx.device)
        slots = np.ascontiguousarray(slots, dtype=np.int32)
        n = slots.size
        masses = np.broadcast_to(np.asarray(masses, dtype=np.float64), (n,)).copy()
        tp = None if tols is None else np.broadcast_to(np.asarray(tols, np.float64), (n,)).copy()
        mp = None if maxiters is None else np.broadcast_to(np.asarray(maxiters, np.int32), (n,)).copy()
        self.ctx._check(self.ctx.lib.wl_engine_admit(
            self.handle, slots.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), n, _ptr(b),
            masses.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
            None if tp is None else tp.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
            None if mp is None else mp.ctypes.data_as(ctypes.POINTER(ctypes.c_int))))
        self._inputs.append(b)

    def step(self, iters: int):
        self.ctx._check(self.ctx.lib.wl_engine_step(self.handle, int(iters)))

    def run(self, max_iters: int):
        """Up to max_iters iterations in one graph launch; stops on the device as soon as a
        slot finishes (asynchronous, like step)."""
        self.ctx._check(self.ctx.lib.wl_engine_run(self.handle, int(max_iters)))

    def poll(self):
        st = np.zeros(self.nslots, dtype=np.int32)
        na = ctypes.c_int()
        self.ctx._check(self.ctx.lib.wl_engine_poll(self.handle, st.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                                    ctypes.byref(na)))
        self._inputs = []
        return st, int(na.value)

    def poll_async(self):
        """Queue the status copies behind the engine's queued work; returns at once."""
        self.ctx._check(self.ctx.lib.wl_engine_poll_async(self.handle))

    def poll_ready(self):
        """(status, n_active) of the last poll_async once its copies have landed, else None.
        Never blocks."""
        st = np.zeros(self.nslots, dtype=np.int32)
        na = ctypes.c_int()
        r = self.ctx.lib.wl_engine_poll_ready(self.handle, st.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                              ctypes.byref(na))
        if r == 0:
            return None
        if r < 0:
            raise WilsonError(WL_ERR_CUDA if r == -2 else WL_ERR_STATE,
                              "wl_engine_poll_ready: " + ("CUDA error" if r == -2 else "no poll queued"))
        self._inputs = []
        return st, int(na.value)

    def retire(self, slot: int, out=None):
        import torch

        if out is None:
            out = torch.empty((*self.ctx.lattice_shape, 4, 3), dtype=torch.complex128, device=self.ctx.device)
        s = WLSolveStats()
        self.ctx._check(self.ctx.lib.wl_engine_retire(self.handle, int(slot), _ptr(out), ctypes.byref(s)))
        return out, dict(iters=s.iters, reliable_updates=s.reliable_updates, status=s.status, true_res=s.true_res)

    @property
    def stream(self):
        """The engine's CUDA stream as a torch ExternalStream."""
        import torch

        return torch.cuda.ExternalStream(int(self.ctx.lib.wl_engine_stream(self.handle)), device=self.ctx.device)

    def debug_apply(self, stage: int, mass: float, x):
        """The engine's iterated-precision operator applied to one field (see
        wl_engine_debug_apply): 0 K_oe, 1 M, 2 M^dag M (EO); 3 D, 4 D^dag D, 5 D^dag (full)."""
        import torch

        x = _c128(x, self.ctx.device)
        out = torch.empty_like(x)
        self.ctx._check(self.ctx.lib.wl_engine_debug_apply(self.handle, int(stage), float(mass), _ptr(x), _ptr(out)))
        return out

    def time_hop(self, reps: int = 20, update: bool = False, cg: bool = False):
        """(ms per launch, algorithmic bytes per launch) of the iterated hop kernel, with
        update=True of the FP64 hop of the reliable update, with cg=True of the fused CG hop
        (which changes the slots' fields: admit them again before stepping)."""
        ms, by = ctypes.c_double(), ctypes.c_double()
        fn = (self.ctx.lib.wl_engine_time_update_hop if update else
              self.ctx.lib.wl_engine_time_cg_hop if cg else self.ctx.lib.wl_engine_time_hop)
        self.ctx._check(fn(self.handle, int(reps), ctypes.byref(ms), ctypes.byref(by)))
        return float(ms.value), float(by.value)

    def close(self):
        if getattr(self, "handle", None) is not None and self.handle.value:
            self.ctx.lib.wl_engine_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
