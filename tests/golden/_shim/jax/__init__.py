"""Numpy-backed stand-in for the small subset of the ``jax`` API that the
jaxQFT Wilson-fermion modules use (test infrastructure only).

It exists so that ``tests/golden/make_golden.py`` can import the reference's
own Python modules (``jaxqft/fermions/wilson.py``, ``jaxqft/models/su3_ym.py``,
``jaxqft/models/su3_wilson_nf2.py``) unchanged and execute their algorithms on
numpy complex128 arrays, producing golden input/output vectors.  Nothing in
the product imports this package.

Semantics kept from JAX:
  * ``jit`` is the identity (tracing changes no values);
  * ``vmap`` maps a Python loop over the given axis and stacks the results;
  * ``scipy.sparse.linalg.cg`` restates JAX's published CG algorithm
    (stopping rule ||r||^2 <= max(tol^2 ||b||^2, atol^2), info=None);
  * ``random`` is a seeded numpy generator (streams differ from threefry by
    design; golden inputs are produced outside the reference anyway).
"""

from __future__ import annotations

import numpy as _np

from . import numpy  # noqa: F401  (jax.numpy)
from . import random  # noqa: F401
from . import scipy  # noqa: F401
from . import lax  # noqa: F401
from . import tree  # noqa: F401

Array = _np.ndarray


def jit(fn=None, **_kw):
    if fn is None:
        return lambda f: f
    return fn


def _stack_results(results):
    first = results[0]
    if isinstance(first, tuple):
        return tuple(_stack_results([r[i] for r in results]) for i in range(len(first)))
    if first is None:
        return None
    return numpy.asarray(_np.stack([_np.asarray(r) for r in results], axis=0))


def vmap(fn, in_axes=0, out_axes=0):
    if out_axes != 0:
        raise NotImplementedError("shim vmap supports out_axes=0 only")

    def mapped(*args):
        axes = in_axes if isinstance(in_axes, (tuple, list)) else (in_axes,) * len(args)
        n = None
        for a, ax in zip(args, axes):
            if ax is not None:
                n = _np.shape(a)[ax]
                break
        if n is None:
            raise ValueError("vmap needs at least one mapped argument")
        outs = []
        for i in range(n):
            call = []
            for a, ax in zip(args, axes):
                if ax is None:
                    call.append(a)
                else:
                    call.append(numpy.asarray(_np.take(a, i, axis=ax)))
            outs.append(fn(*call))
        return _stack_results(outs)

    return mapped


def grad(*_a, **_k):
    raise NotImplementedError("autodiff is not available in the numpy shim")


def block_until_ready(x):
    return x


def device_put(x, *_a, **_kw):
    """No device: the array itself (as jax.device_put onto the CPU backend)."""
    return numpy.asarray(x)
