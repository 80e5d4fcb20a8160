"""jax.numpy.fft stand-in (same transform definitions as numpy.fft)."""

import numpy as _np

from .._core import wrap


def fft(a, n=None, axis=-1, norm=None):
    return wrap(_np.fft.fft(_np.asarray(a), n=n, axis=axis, norm=norm))


def ifft(a, n=None, axis=-1, norm=None):
    return wrap(_np.fft.ifft(_np.asarray(a), n=n, axis=axis, norm=norm))


def rfft(a, n=None, axis=-1, norm=None):
    return wrap(_np.fft.rfft(_np.asarray(a), n=n, axis=axis, norm=norm))


def irfft(a, n=None, axis=-1, norm=None):
    return wrap(_np.fft.irfft(_np.asarray(a), n=n, axis=axis, norm=norm))
