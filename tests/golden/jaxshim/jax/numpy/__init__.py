"""jax.numpy stand-in: NumPy functions returning ShimArray (fixture generation)."""

import numpy as _np

from .._core import ShimArray, _strip, wrap
from . import fft  # noqa: F401

ndarray = _np.ndarray
pi = _np.pi
inf = _np.inf
nan = _np.nan
float32 = _np.float32
float64 = _np.float64
complex64 = _np.complex64
complex128 = _np.complex128
int32 = _np.int32
int64 = _np.int64
bool_ = _np.bool_
newaxis = None


def _wrapfn(f):
    def g(*a, **kw):
        _strip(kw)
        return wrap(f(*a, **kw))

    g.__name__ = getattr(f, "__name__", "fn")
    return g


def sum(a, axis=None, dtype=None, **kw):  # noqa: A001
    _strip(kw)
    a = _np.asarray(a)
    if dtype is not None and _np.iscomplexobj(a) and not _np.issubdtype(
        _np.dtype(dtype), _np.complexfloating
    ):
        a = a.real
    return wrap(_np.sum(a, axis=axis, dtype=dtype, **kw))


def zeros(shape, dtype=None, **kw):
    _strip(kw)
    return wrap(_np.zeros(shape, dtype=float if dtype is None else dtype))


def ones(shape, dtype=None, **kw):
    _strip(kw)
    return wrap(_np.ones(shape, dtype=float if dtype is None else dtype))


def array(x, dtype=None, **kw):
    _strip(kw)
    return wrap(_np.array(x, dtype=dtype))


def asarray(x, dtype=None, **kw):
    _strip(kw)
    return wrap(_np.array(x, dtype=dtype))


def iscomplexobj(x):
    return _np.iscomplexobj(x)


def result_type(*a):
    return _np.result_type(*a)


def __getattr__(name):
    f = getattr(_np, name)
    if callable(f):
        return _wrapfn(f)
    return f
