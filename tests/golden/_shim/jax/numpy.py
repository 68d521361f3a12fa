"""``jax.numpy`` stand-in: numpy plus functional ``x.at[idx].set(v)`` updates."""

from __future__ import annotations

import numpy as _np
from numpy import *  # noqa: F401,F403
from numpy import linalg  # noqa: F401


class _AtIndexer:
    def __init__(self, arr):
        self._arr = arr

    def __getitem__(self, idx):
        return _AtSetter(self._arr, idx)


class _AtSetter:
    def __init__(self, arr, idx):
        self._arr = arr
        self._idx = idx

    def set(self, value, **_kw):
        out = _np.array(self._arr, copy=True).view(ShimArray)
        out[self._idx] = value
        return out

    def add(self, value, **_kw):
        out = _np.array(self._arr, copy=True).view(ShimArray)
        _np.add.at(out, self._idx, value)
        return out


class ShimArray(_np.ndarray):
    """ndarray with JAX's ``.at`` functional-update property and a no-op
    ``block_until_ready``."""

    @property
    def at(self):
        return _AtIndexer(self)

    def block_until_ready(self):
        return self


def _wrap(x):
    if isinstance(x, _np.ndarray):
        return x.view(ShimArray)
    return x


def asarray(x, dtype=None):
    return _wrap(_np.asarray(x, dtype=dtype))


def array(x, dtype=None, **kw):
    return _wrap(_np.array(x, dtype=dtype, **kw))


def zeros(shape, dtype=float):
    return _wrap(_np.zeros(shape, dtype=dtype))


def zeros_like(x, dtype=None):
    return _wrap(_np.zeros_like(x, dtype=dtype))


def ones(shape, dtype=float):
    return _wrap(_np.ones(shape, dtype=dtype))


def einsum(*args, **kw):
    kw.setdefault("optimize", True)
    return _wrap(_np.einsum(*args, **kw))


def take(a, indices, axis=None, **_kw):
    return _wrap(_np.take(a, indices, axis=axis))


def stack(arrays, axis=0):
    return _wrap(_np.stack(arrays, axis=axis))


def roll(a, shift, axis=None):
    return _wrap(_np.roll(a, shift, axis=axis))


def broadcast_to(a, shape):
    return _wrap(_np.broadcast_to(a, shape))


ndarray = _np.ndarray
