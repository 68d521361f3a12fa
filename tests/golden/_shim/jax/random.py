"""``jax.random`` stand-in backed by numpy's PCG64 (streams differ from JAX)."""

from __future__ import annotations

import numpy as _np


def PRNGKey(seed):
    return _np.array([int(seed) & 0xFFFFFFFF, 0], dtype=_np.uint64)


def _rng(key):
    return _np.random.default_rng([int(k) for k in _np.asarray(key).ravel()])


def split(key, num=2):
    words = _rng(key).integers(0, 2**32, size=(num, 2), dtype=_np.uint64)
    return words


def normal(key, shape=(), dtype=_np.float32):
    return _rng(key).standard_normal(shape).astype(dtype)


def uniform(key, shape=(), dtype=_np.float32, minval=0.0, maxval=1.0):
    return (_rng(key).random(shape) * (maxval - minval) + minval).astype(dtype)
