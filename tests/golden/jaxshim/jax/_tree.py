"""Pytree helpers for the NumPy stand-in of ``jax`` (test infrastructure only).

Dataclass fields flagged ``static`` in their metadata are not leaves; ``None``
is an empty subtree, as in JAX.
"""
from __future__ import annotations

import dataclasses

import numpy as _np


def _is_namedtuple(x):
    return isinstance(x, tuple) and hasattr(x, "_fields")


def _children(x):
    """Return (kind, children, rebuild) or None when x is a leaf."""
    if x is None:
        return ("none", [], lambda ch: None)
    if dataclasses.is_dataclass(x) and not isinstance(x, type):
        names = [f.name for f in dataclasses.fields(x) if not f.metadata.get("static", False)]
        vals = [getattr(x, n) for n in names]

        def rebuild(ch, x=x, names=names):
            return dataclasses.replace(x, **dict(zip(names, ch)))
        return ("dc", vals, rebuild)
    if _is_namedtuple(x):
        return ("nt", list(x), lambda ch, t=type(x): t(*ch))
    if isinstance(x, (tuple, list)):
        return ("seq", list(x), lambda ch, t=type(x): t(ch))
    if isinstance(x, dict):
        keys = sorted(x.keys())
        return ("dict", [x[k] for k in keys], lambda ch, keys=keys: dict(zip(keys, ch)))
    return None


def tree_flatten(x):
    leaves = []

    def rec(v):
        c = _children(v)
        if c is None:
            leaves.append(v)
            return ("leaf",)
        kind, ch, rebuild = c
        return (kind, rebuild, [rec(e) for e in ch])
    spec = rec(x)
    return leaves, spec


def tree_unflatten(spec, leaves):
    it = iter(leaves)

    def rec(s):
        if s[0] == "leaf":
            return next(it)
        _, rebuild, subs = s
        return rebuild([rec(e) for e in subs])
    return rec(spec)


def tree_leaves(x):
    return tree_flatten(x)[0]


def tree_map(f, x, *rest):
    leaves, spec = tree_flatten(x)
    others = [tree_flatten(r)[0] for r in rest]
    out = [f(l, *[o[i] for o in others]) for i, l in enumerate(leaves)]
    return tree_unflatten(spec, out)
