"""Thread-parallel slices for the oracle (test and baseline infrastructure
only).

With the default of one thread every helper makes exactly the serial call it
wraps.  With more threads it splits the call into independent slices along
an axis the operation does not mix: lines of an FFT, modes of a y-stencil
or of a banded solve.  It runs the slices on a thread pool and concatenates
the results.  Each slice computes its lines or modes exactly as the whole
call does, so the results are bitwise identical
(``tests/test_oracle_parallel.py``).  NumPy releases the GIL inside its FFT,
einsum and array loops, which is what the threads use.
"""

from __future__ import annotations

from concurrent.futures import ThreadPoolExecutor

import numpy as np

_threads = 1
_pool: ThreadPoolExecutor | None = None

# The banded solve's per-step loop is short NumPy calls on a slice of modes;
# beyond about four threads the interpreter lock, not the arithmetic, limits
# it, so it uses at most this many.
SOLVE_THREADS_MAX = 4


def set_threads(n: int) -> None:
    """Use n threads (n = 1: the serial calls)."""
    global _threads, _pool
    n = max(1, int(n))
    if _pool is not None:
        _pool.shutdown(wait=True)
        _pool = None
    _threads = n
    if n > 1:
        _pool = ThreadPoolExecutor(max_workers=n)


def threads() -> int:
    return _threads


def split(fn, arrays, axis: int, n: int | None = None):
    """fn(*slices) over n slices of every array along ``axis``, concatenated
    along the same axis of the result."""
    n = _threads if n is None else min(n, _threads)
    size = arrays[0].shape[axis]
    n = min(n, size // 2)  # slices of at least two rows
    if n <= 1 or _pool is None:
        return fn(*arrays)
    edges = np.linspace(0, size, n + 1).astype(int)

    def part(k):
        cut = slice(edges[k], edges[k + 1])
        return fn(*(a[(slice(None),) * axis + (cut,)] for a in arrays))

    return np.concatenate(list(_pool.map(part, range(n))), axis=axis)


def fft(fn, x: np.ndarray, axis: int, **kw) -> np.ndarray:
    """``fn(x, axis=axis, **kw)`` (a numpy.fft transform), split along another
    axis: every 1-D line is transformed on its own."""
    other = 0 if axis % x.ndim != 0 else 1
    return split(lambda a: fn(a, axis=axis, **kw), (x,), other)


def einsum_y(D: np.ndarray, u: np.ndarray) -> np.ndarray:
    """``einsum("ij,...j->...i", D, u)``: the y-stencil of every mode, split
    over the leading (mode) axis."""
    return split(lambda a: np.einsum("ij,zxj->zxi", D, a), (u,), 0)
