"""jax.lax stand-in: scan and dynamic slices (fixture generation)."""

import numpy as _np

from ._core import wrap


def scan(f, init, xs, length=None):
    carry = init
    ys = []
    for x in (xs if xs is not None else range(length)):
        carry, y = f(carry, x)
        ys.append(y)
    if ys and ys[0] is not None:
        return carry, wrap(_np.stack(ys))
    return carry, None


def dynamic_slice_in_dim(x, start, size, axis=0):
    x = _np.asarray(x)
    start = int(start)
    idx = [slice(None)] * x.ndim
    idx[axis] = slice(start, start + size)
    return wrap(x[tuple(idx)])


def dynamic_update_slice_in_dim(x, upd, start, axis=0):
    out = _np.array(x, copy=True)
    upd = _np.asarray(upd)
    start = int(start)
    idx = [slice(None)] * out.ndim
    idx[axis] = slice(start, start + upd.shape[axis])
    out[tuple(idx)] = upd
    return wrap(out)
