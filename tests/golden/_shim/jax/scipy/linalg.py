"""``jax.scipy.linalg.expm`` via scipy (batched over leading axes)."""

from __future__ import annotations

import numpy as _np
import scipy.linalg as _sl

from jax.numpy import asarray as _asarray


def expm(a):
    return _asarray(_sl.expm(_np.asarray(a)))
