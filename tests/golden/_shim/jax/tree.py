"""``jax.tree`` stand-in for single-array pytrees."""

from __future__ import annotations


def map(fn, tree, *rest):
    return fn(tree, *rest)
