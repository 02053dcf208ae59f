"""NumPy-backed stand-in for ``jax.numpy`` used only to execute the reference
IBIS step in this container (no jaxlib is installed) so that golden fixtures
can be generated from the reference's own source.

Arrays are ``JArr`` (an ndarray subclass) so that the functional update
syntax ``x.at[idx].set(v)`` works.  Integer powers with a Python-int exponent
are evaluated by repeated squaring, which is how XLA lowers ``integer_pow``.
Test infrastructure only: never imported by the product.
"""
from __future__ import annotations

import builtins
import numpy as _np


class _AtIndexer:
    __slots__ = ("_arr", "_idx")

    def __init__(self, arr, idx):
        self._arr = arr
        self._idx = idx

    def _apply(self, fn):
        out = _np.array(self._arr, copy=True)
        fn(out)
        return out.view(JArr)

    def set(self, v):
        def f(o):
            o[self._idx] = _np.asarray(v)
        return self._apply(f)

    def add(self, v):
        def f(o):
            o[self._idx] = o[self._idx] + _np.asarray(v)
        return self._apply(f)

    def multiply(self, v):
        def f(o):
            o[self._idx] = o[self._idx] * _np.asarray(v)
        return self._apply(f)

    mul = multiply

    def min(self, v):
        def f(o):
            o[self._idx] = _np.minimum(o[self._idx], _np.asarray(v))
        return self._apply(f)

    def max(self, v):
        def f(o):
            o[self._idx] = _np.maximum(o[self._idx], _np.asarray(v))
        return self._apply(f)

    def get(self):
        return self._arr[self._idx]


class _At:
    __slots__ = ("_arr",)

    def __init__(self, arr):
        self._arr = arr

    def __getitem__(self, idx):
        return _AtIndexer(self._arr, idx)


def _ipow(x, n):
    """x**n for a non-negative Python int n by repeated squaring."""
    if n == 0:
        return _np.ones_like(_np.asarray(x))
    result = None
    base = _np.asarray(x)
    while n:
        if n & 1:
            result = base if result is None else result * base
        n >>= 1
        if n:
            base = base * base
    return result


class JArr(_np.ndarray):
    @property
    def at(self):
        return _At(self)

    def block_until_ready(self):
        return self

    def __pow__(self, other):
        if isinstance(other, (int, _np.integer)) and not isinstance(other, bool):
            n = int(other)
            if n >= 0:
                return _wrap(_ipow(_np.asarray(self), n))
            return _wrap(1.0 / _ipow(_np.asarray(self), -n))
        return _wrap(_np.power(_np.asarray(self), _np.asarray(other)))

    def __rpow__(self, other):
        return _wrap(_np.power(_np.asarray(other), _np.asarray(self)))


def _wrap(x):
    if isinstance(x, _np.ndarray):
        return x.view(JArr)
    if isinstance(x, (_np.generic, float, int, bool)):
        return _np.asarray(x).view(JArr)
    if isinstance(x, tuple):
        return tuple(_wrap(v) for v in x)
    if isinstance(x, list):
        return [_wrap(v) for v in x]
    return x


# dtypes and constants
float16 = _np.float16
float32 = _np.float32
float64 = _np.float64
int8 = _np.int8
int16 = _np.int16
int32 = _np.int32
int64 = _np.int64
uint8 = _np.uint8
uint32 = _np.uint32
bool_ = _np.bool_
floating = _np.floating
integer = _np.integer
ndarray = _np.ndarray
pi = _np.pi
inf = _np.inf
nan = _np.nan
newaxis = None
e = _np.e
dtype = _np.dtype
issubdtype = _np.issubdtype
ndim = _np.ndim
shape = _np.shape
finfo = _np.finfo
iinfo = _np.iinfo


def array(x, dtype=None, copy=True):
    return _np.array(x, dtype=dtype).view(JArr)


def asarray(x, dtype=None):
    return _np.asarray(x, dtype=dtype).view(JArr)


def where(c, a=None, b=None):
    if a is None and b is None:
        return _wrap(_np.where(c))
    return _wrap(_np.where(c, a, b))


def clip(x, a_min=None, a_max=None, **kw):
    lo = kw.pop("min", a_min)
    hi = kw.pop("max", a_max)
    x = _np.asarray(x)
    if lo is not None:
        x = _np.maximum(x, lo)
    if hi is not None:
        x = _np.minimum(x, hi)
    return _wrap(x)


def power(a, b):
    if isinstance(b, (int, _np.integer)) and not isinstance(b, bool) and int(b) >= 0:
        return _wrap(_ipow(a, int(b)))
    return _wrap(_np.power(a, b))


def round(x, decimals=0):
    return _wrap(_np.round(x, decimals))


def sum(x, axis=None, keepdims=False, dtype=None):
    return _wrap(_np.sum(x, axis=axis, keepdims=keepdims, dtype=dtype))


def __getattr__(name):
    obj = getattr(_np, name)
    if callable(obj) and not isinstance(obj, type):
        def wrapped(*a, **k):
            return _wrap(obj(*a, **k))
        wrapped.__name__ = name
        return wrapped
    return obj


class linalg:
    @staticmethod
    def solve(a, b):
        return _wrap(_np.linalg.solve(a, b))


def zeros(shape, dtype=None):
    return _np.zeros(shape, dtype=dtype if dtype is not None else _np.float64).view(JArr)


def ones(shape, dtype=None):
    return _np.ones(shape, dtype=dtype if dtype is not None else _np.float64).view(JArr)


def full(shape, fill_value, dtype=None):
    if dtype is None:
        fv = _np.asarray(fill_value)
        dtype = fv.dtype if fv.dtype.kind in "fc" else (_np.float64 if fv.dtype.kind != "b" and fv.dtype.kind != "i" else fv.dtype)
    return _np.full(shape, fill_value, dtype=dtype).view(JArr)


def zeros_like(x, dtype=None):
    return _np.zeros_like(_np.asarray(x), dtype=dtype).view(JArr)


def ones_like(x, dtype=None):
    return _np.ones_like(_np.asarray(x), dtype=dtype).view(JArr)


def full_like(x, v, dtype=None):
    return _np.full_like(_np.asarray(x), v, dtype=dtype).view(JArr)


_ = builtins
