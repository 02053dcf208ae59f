"""Minimal NumPy-backed stand-in for ``jax`` (test infrastructure only).

Provides just enough of the API (``numpy``, ``lax.scan``, ``lax.fori_loop``,
``tree.map``, ``jit``) for the reference IBIS hourly step to execute eagerly
in float64 in a container without jaxlib, so that golden fixtures can be
produced from the reference's own code.
"""
from __future__ import annotations

import types as _types

import numpy as _onp

from . import numpy  # noqa: F401
from .numpy import JArr as Array  # noqa: F401
from . import _tree

__version__ = "0.0-numpy-shim"


class _Config:
    def update(self, *a, **k):
        return None

    jax_enable_x64 = True


config = _Config()


def jit(fn=None, **kw):
    if fn is None:
        return lambda f: f
    return fn


def vmap(fn, in_axes=0, out_axes=0):
    def wrapped(*args):
        n = None
        for a in args:
            if isinstance(a, _onp.ndarray):
                n = a.shape[0]
                break
        outs = [fn(*[a[i] if isinstance(a, _onp.ndarray) else a for a in args]) for i in range(n)]
        return _tree.tree_map(lambda *xs: numpy.stack(xs), *outs)
    return wrapped


def grad(*a, **k):
    raise NotImplementedError("gradients are not available in the numpy shim")


def block_until_ready(x):
    return x


def _scan(f, init, xs=None, length=None, reverse=False, unroll=1):
    if xs is None:
        n = length
        seq = [None] * n
    else:
        leaves = _tree.tree_leaves(xs)
        n = leaves[0].shape[0]
        seq = [_tree.tree_map(lambda a: a[i], xs) for i in range(n)]
    idx = range(n - 1, -1, -1) if reverse else range(n)
    carry = init
    ys = []
    for i in idx:
        carry, y = f(carry, seq[i])
        ys.append(y)
    if reverse:
        ys = ys[::-1]
    if ys and ys[0] is not None:
        stacked = _tree.tree_map(lambda *a: numpy.stack(a), *ys)
    else:
        stacked = None
    return carry, stacked


def _fori_loop(lo, hi, body, init):
    v = init
    for i in range(int(lo), int(hi)):
        v = body(i, v)
    return v


def _cond(pred, tf, ff, *ops):
    return tf(*ops) if bool(pred) else ff(*ops)


def _select(c, a, b):
    return numpy.where(c, a, b)


lax = _types.SimpleNamespace(scan=_scan, fori_loop=_fori_loop, cond=_cond, select=_select,
                             stop_gradient=lambda x: x)

tree = _types.SimpleNamespace(map=_tree.tree_map, leaves=_tree.tree_leaves,
                              flatten=_tree.tree_flatten, unflatten=_tree.tree_unflatten)
tree_util = _types.SimpleNamespace(tree_map=_tree.tree_map, tree_leaves=_tree.tree_leaves,
                                   tree_flatten=_tree.tree_flatten)


class _Random(_types.SimpleNamespace):
    pass


def _key(seed):
    return numpy.asarray(_onp.array([0, int(seed)], dtype=_onp.uint32))


def _split(key, num=2):
    k = _onp.asarray(key).astype(_onp.uint64)
    out = _onp.stack([(k * 6364136223846793005 + i + 1) % (2 ** 32) for i in range(num)]).astype(_onp.uint32)
    return numpy.asarray(out)


random = _Random(PRNGKey=_key, key=_key, split=_split)
