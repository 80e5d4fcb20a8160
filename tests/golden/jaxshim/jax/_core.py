"""Array type for the NumPy-backed jax stand-in (golden-fixture generation)."""

import numpy as _np


class ShimArray(_np.ndarray):
    """ndarray with JAX's functional ``.at[...]`` update syntax."""

    @property
    def at(self):
        return _At(self)


class _At:
    def __init__(self, arr):
        self._arr = arr

    def __getitem__(self, idx):
        return _AtIdx(self._arr, idx)


def _strip(kw):
    kw.pop("out_sharding", None)
    kw.pop("mode", None)
    kw.pop("indices_are_sorted", None)
    kw.pop("unique_indices", None)
    return kw


class _AtIdx:
    def __init__(self, arr, idx):
        self._arr = arr
        self._idx = idx

    def _new(self, values):
        out = _np.array(self._arr, copy=True)
        v = _np.asarray(values)
        if _np.iscomplexobj(v) and not _np.iscomplexobj(out):
            out = out.astype(_np.result_type(out, v))
        return out, v

    def set(self, values, **kw):
        _strip(kw)
        out, v = self._new(values)
        out[self._idx] = v
        return wrap(out)

    def add(self, values, **kw):
        _strip(kw)
        out, v = self._new(values)
        out[self._idx] = out[self._idx] + v
        return wrap(out)

    def subtract(self, values, **kw):
        _strip(kw)
        out, v = self._new(values)
        out[self._idx] = out[self._idx] - v
        return wrap(out)

    def multiply(self, values, **kw):
        _strip(kw)
        out, v = self._new(values)
        out[self._idx] = out[self._idx] * v
        return wrap(out)

    def get(self, **kw):
        _strip(kw)
        return wrap(_np.asarray(self._arr)[self._idx])


def wrap(x):
    if isinstance(x, tuple):
        return tuple(wrap(v) for v in x)
    if isinstance(x, list):
        return [wrap(v) for v in x]
    if isinstance(x, _np.ndarray):
        return x.view(ShimArray)
    if isinstance(x, (_np.generic, float, int, complex, bool)):
        return _np.asarray(x).view(ShimArray)
    return x
