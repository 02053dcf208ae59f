"""Minimal stand-in for ``equinox`` (test infrastructure only).

``Module`` subclasses become frozen dataclasses; ``field(static=True)`` marks a
non-leaf field; ``tree_at`` rebuilds a pytree with the nodes that a selector
lambda reaches replaced.
"""
from __future__ import annotations

import dataclasses

import numpy as _np


def field(*, static=False, default=dataclasses.MISSING, default_factory=dataclasses.MISSING,
          converter=None, **kw):
    md = {"static": bool(static)}
    if converter is not None:
        md["converter"] = converter
    if default is not dataclasses.MISSING:
        return dataclasses.field(default=default, metadata=md)
    if default_factory is not dataclasses.MISSING:
        return dataclasses.field(default_factory=default_factory, metadata=md)
    return dataclasses.field(metadata=md)


class Module:
    def __init_subclass__(cls, **kw):
        super().__init_subclass__(**kw)
        # mutable array defaults are not allowed by dataclasses; wrap them
        for name, val in list(cls.__dict__.items()):
            if name.startswith("__"):
                continue
            ann = cls.__dict__.get("__annotations__", {})
            if name in ann and isinstance(val, _np.ndarray):
                setattr(cls, name, dataclasses.field(default_factory=lambda v=val: v))
        dataclasses.dataclass(frozen=True, eq=False, repr=False)(cls)
        return cls


def filter_jit(fn=None, **kw):
    if fn is None:
        return lambda f: f
    return fn


class _Path:
    """Records attribute / index access made by a tree_at selector."""

    def __init__(self, path=()):
        object.__setattr__(self, "_path", path)

    def __getattr__(self, name):
        if name.startswith("__"):
            raise AttributeError(name)
        return _Path(self._path + (("attr", name),))

    def __getitem__(self, key):
        return _Path(self._path + (("item", key),))


def _get(node, step):
    kind, key = step
    return getattr(node, key) if kind == "attr" else node[key]


def _set(node, step, value):
    kind, key = step
    if kind == "attr":
        if hasattr(node, "_replace") and hasattr(node, "_fields"):
            return node._replace(**{key: value})
        return dataclasses.replace(node, **{key: value})
    if isinstance(node, tuple):
        lst = list(node)
        lst[key] = value
        return type(node)(*lst) if hasattr(node, "_fields") else tuple(lst)
    if isinstance(node, list):
        lst = list(node)
        lst[key] = value
        return lst
    if isinstance(node, dict):
        d = dict(node)
        d[key] = value
        return d
    raise TypeError(f"tree_at cannot set {kind} {key!r} on {type(node)}")


def _replace_path(root, path, value):
    if not path:
        return value
    child = _get(root, path[0])
    return _set(root, path[0], _replace_path(child, path[1:], value))


def tree_at(where, pytree, replace=None, replace_fn=None, is_leaf=None):
    sel = where(_Path())
    multi = isinstance(sel, (tuple, list))
    paths = [s._path for s in sel] if multi else [sel._path]
    if replace_fn is not None:
        vals = []
        for p in paths:
            node = pytree
            for st in p:
                node = _get(node, st)
            vals.append(replace_fn(node))
    else:
        vals = list(replace) if multi else [replace]
    out = pytree
    for p, v in zip(paths, vals):
        out = _replace_path(out, p, v)
    return out
