"""``jax.scipy.sparse`` stand-in."""

from . import linalg  # noqa: F401
