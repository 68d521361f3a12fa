"""ctypes binding of the C/OpenMP CPU oracle (oracle/c/wilson_cpu.c).

TEST INFRASTRUCTURE ONLY: used by tests and by bench.py's CPU-baseline legs.
"""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libwilson_cpu.so")


def build(force: bool = False) -> str:
    src = os.path.join(HERE, "c", "wilson_cpu.c")
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-B" if force else "-s", "-C", os.path.join(HERE, "c")], check=True)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        vp, i, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        L.wcpu_create.restype = vp
        L.wcpu_create.argtypes = [vp, vp, vp, vp, d]
        L.wcpu_destroy.argtypes = [vp]
        L.wcpu_normal.argtypes = [vp, vp, vp]
        L.wcpu_hop.argtypes = [vp, i, i, vp, vp]
        L.wcpu_cg.restype = i
        L.wcpu_cg.argtypes = [vp, vp, vp, d, i, ctypes.POINTER(d)]
        L.wcpu_threads.restype = i
        _lib = L
    return _lib


class CpuWilson:
    """FP64 even-odd normal operator M^dag M and CG on one configuration."""

    def __init__(self, U, shape, bc, mass):
        self.U = np.ascontiguousarray(U, dtype=np.complex128)  # [4, *shape, 3, 3]
        self.shape = tuple(int(v) for v in shape)
        dims = np.asarray(self.shape, dtype=np.int32)
        bcs = np.asarray([complex(np.complex64(complex(b))) for b in bc])
        self._re = np.ascontiguousarray(bcs.real)
        self._im = np.ascontiguousarray(bcs.imag)
        self.h = lib().wcpu_create(dims.ctypes.data, self._re.ctypes.data, self._im.ctypes.data, self.U.ctypes.data,
                                   float(mass))
        self.vh = int(np.prod(self.shape)) // 2
        self.m0 = float(mass) + 4.0

    def normal(self, x):
        x = np.ascontiguousarray(x, dtype=np.complex128)
        out = np.empty_like(x)
        lib().wcpu_normal(self.h, x.ctypes.data, out.ctypes.data)
        return out

    def hop(self, target, sign, x):
        """K x on compact fields: the target-parity sites of -1/2 sum_mu of the
        hops of D (sign -1) or D^dag (sign +1) from the other parity's x."""
        x = np.ascontiguousarray(x, dtype=np.complex128)
        out = np.empty_like(x)
        lib().wcpu_hop(self.h, int(target), int(sign), x.ctypes.data, out.ctypes.data)
        return out

    def apply_D(self, psi, dag=False):
        """D (or D^dag) on one reference-layout field [*shape, 4, 3], from the
        compact hops: (D x)_p = m0 x_p + K_{p,1-p} x_{1-p}."""
        from oracle import wilson as W

        sign = 1 if dag else -1
        m0 = float(self.m0)
        xe, xo = W.pack(psi[None], 0)[0], W.pack(psi[None], 1)[0]
        out_e = m0 * xe + self.hop(0, sign, xo)
        out_o = m0 * xo + self.hop(1, sign, xe)
        return W.unpack(out_e[None], self.shape, 0)[0] + W.unpack(out_o[None], self.shape, 1)[0]

    def cg(self, b, tol, maxiter):
        b = np.ascontiguousarray(b, dtype=np.complex128)
        x = np.empty_like(b)
        res = ctypes.c_double()
        k = lib().wcpu_cg(self.h, b.ctypes.data, x.ctypes.data, float(tol), int(maxiter), ctypes.byref(res))
        return x, int(k), float(res.value)

    def __del__(self):
        try:
            lib().wcpu_destroy(self.h)
        except Exception:
            pass


def threads() -> int:
    return int(lib().wcpu_threads())
