"""NumPy-backed stand-in for the jax API subset used by the reference solver.

Only for generating golden fixtures from the reference's own source in a
container without JAX (tests/golden/make_golden.py).  One CPU device,
float64, eager execution: ``jit`` is the identity, ``vmap`` loops,
``shard_map``/``reshard`` are no-ops.
"""

import numpy as _np

from . import lax, numpy, scipy, sharding, tree_util  # noqa: F401
from ._core import ShimArray, wrap

Array = _np.ndarray


class _Config:
    def update(self, *a, **kw):
        return None


config = _Config()


class _Distributed:
    def initialize(self, *a, **kw):
        return None


distributed = _Distributed()


class _Device:
    def __repr__(self):
        return "CpuDevice(id=0)"


def devices():
    return [_Device()]


def process_index():
    return 0


def make_mesh(shape, axis_names=None, axis_types=None):
    return ("mesh", tuple(shape), axis_names)


def set_mesh(mesh):
    return None


def device_put(x, sharding=None):
    return wrap(_np.asarray(x))


def make_array_from_callback(shape, sharding, cb):
    return wrap(_np.asarray(cb(tuple(slice(0, n, None) for n in shape))))


def block_until_ready(x):
    return x


def jit(f=None, **kw):
    if f is None:
        return lambda g: g
    return f


def shard_map(f, mesh=None, in_specs=None, out_specs=None, **kw):
    return f


def _stack(outs):
    if isinstance(outs[0], tuple):
        return tuple(_stack([o[i] for o in outs]) for i in range(len(outs[0])))
    return wrap(_np.stack([_np.asarray(o) for o in outs]))


def vmap(f, in_axes=0, out_axes=0):
    def g(*args):
        axes = in_axes if isinstance(in_axes, (tuple, list)) else (in_axes,) * len(args)
        n = None
        for a, ax in zip(args, axes):
            if ax is not None:
                n = _np.asarray(a).shape[ax] if not isinstance(a, tuple) else len(a[0])
                break
        outs = []
        for i in range(n):
            sub = []
            for a, ax in zip(args, axes):
                if ax is None:
                    sub.append(a)
                elif isinstance(a, tuple):
                    sub.append(tuple(wrap(_np.take(_np.asarray(t), i, axis=ax)) for t in a))
                else:
                    sub.append(wrap(_np.take(_np.asarray(a), i, axis=ax)))
            outs.append(f(*sub))
        return _stack(outs)

    return g
