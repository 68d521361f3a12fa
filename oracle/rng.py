"""numpy restatement of the device random fields (jaxqft_b200/csrc/wl_rng.cuh).

TEST INFRASTRUCTURE ONLY (the GPU tests compare the kernels with it).

Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
as 1, 2, 3", SC 2011) on vectors of counters, 53-bit uniforms in (0, 1) from
two output words, Box-Muller normals, and the two fields built from them: the
complex Gaussian spinor of random_fermion (jaxqft/models/su3_wilson_nf2.py:
1169-1175) and the su(3) algebra draw of _sample_algebra (jaxqft/models/
su3_ym.py:238-244).
"""

from __future__ import annotations

import numpy as np

M0, M1 = np.uint64(0xD2511F53), np.uint64(0xCD9E8D57)
W0, W1 = 0x9E3779B9, 0xBB67AE85
MASK = np.uint64(0xFFFFFFFF)


def philox4x32_10(c0, c1, c2, c3, k0: int, k1: int):
    c = [np.asarray(v, dtype=np.uint64) & MASK for v in (c0, c1, c2, c3)]
    for _ in range(10):
        p0 = M0 * c[0]
        p1 = M1 * c[2]
        hi0, lo0 = p0 >> np.uint64(32), p0 & MASK
        hi1, lo1 = p1 >> np.uint64(32), p1 & MASK
        c = [hi1 ^ c[1] ^ np.uint64(k0), lo1, hi0 ^ c[3] ^ np.uint64(k1), lo0]
        k0 = (k0 + W0) & 0xFFFFFFFF
        k1 = (k1 + W1) & 0xFFFFFFFF
    return c


def u01(a, b):
    x = ((a << np.uint64(32)) | b) >> np.uint64(11)
    return (x.astype(np.float64) + 0.5) * 2.0 ** -53


def normal2(seed: int, stream: int, ctr, field: int):
    c = philox4x32_10(ctr, np.full_like(ctr, field), np.full_like(ctr, stream & 0xFFFFFFFF),
                      np.full_like(ctr, (stream >> 32) & 0xFFFFFFFF), seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF)
    u, v = u01(c[0], c[1]), u01(c[2], c[3])
    r = np.sqrt(-2.0 * np.log(u))
    return r * np.cos(2.0 * np.pi * v), r * np.sin(2.0 * np.pi * v)


def random_spinor(seed: int, stream: int, n: int, volume: int):
    """[n, volume, 4, 3] complex: (g0 + i g1) / sqrt(2) per component."""
    out = np.empty((n, volume * 12), dtype=np.complex128)
    ctr = np.arange(volume * 12, dtype=np.uint64)
    for f in range(n):
        g0, g1 = normal2(seed, stream, ctr, f)
        out[f] = (g0 + 1j * g1) / np.sqrt(2.0)
    return out.reshape(n, volume, 4, 3)


def random_algebra(seed: int, stream: int, batch: int, volume: int, scale: float = 1.0):
    """[batch, 4 * volume, 3, 3] complex: TA(scale (G1 + i G2)) per link."""
    ctr = np.arange(4 * volume * 9, dtype=np.uint64)
    out = np.empty((batch, 4 * volume, 3, 3), dtype=np.complex128)
    for f in range(batch):
        g0, g1 = normal2(seed, stream, ctr, f)
        x = (scale * (g0 + 1j * g1)).reshape(4 * volume, 3, 3)
        y = 0.5 * (x - np.conj(np.swapaxes(x, -1, -2)))
        tr = np.trace(y, axis1=-2, axis2=-1) / 3.0
        out[f] = y - tr[:, None, None] * np.eye(3)
    return out
