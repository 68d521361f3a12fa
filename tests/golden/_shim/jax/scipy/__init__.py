"""``jax.scipy`` stand-in."""

from . import linalg  # noqa: F401
from . import sparse  # noqa: F401
