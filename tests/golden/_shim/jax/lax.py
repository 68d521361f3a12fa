"""``jax.lax`` stand-in (Python control flow)."""

from __future__ import annotations


def while_loop(cond_fun, body_fun, init_val):
    val = init_val
    while cond_fun(val):
        val = body_fun(val)
    return val


def scan(f, init, xs, length=None):
    raise NotImplementedError("lax.scan is not provided by the numpy shim")
