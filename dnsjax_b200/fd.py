"""Finite-difference weights on the Chebyshev-Gauss-Lobatto grid (host setup).

Same construction as the reference (``src/dnsjax/fd.py:21-108``): Fornberg's
(1998) recurrence for the weights, ``p+1``-point stencils for D1 and
``p+2``-point stencils for D2, centred in the interior and shifted to stay
inside the domain near the walls.  Returned both dense (for host-side
setup) and as compact bands (``j0`` start column and weights per row) for
the CUDA kernels.
"""

from __future__ import annotations

import numpy as np


def fornberg_weights(z: float, x: np.ndarray, m: int) -> np.ndarray:
    """Weights ``w[j, d]`` of the d-th derivative at ``z`` on nodes ``x``.

    Fornberg, SIAM Rev. 40 (1998) 685-691: the weights for ``n+1`` nodes
    are built from those for ``n`` nodes, one new node at a time.
    """
    npts = len(x)
    w = np.zeros((npts, m + 1))
    w[0, 0] = 1.0
    prod_prev = 1.0
    dz_last = x[0] - z
    for i in range(1, npts):
        top = min(i, m)
        prod = 1.0
        dz_prev = dz_last
        dz_last = x[i] - z
        for j in range(i):
            gap = x[i] - x[j]
            prod *= gap
            if j == i - 1:
                for d in range(top, 0, -1):
                    w[i, d] = prod_prev * (d * w[i - 1, d - 1]
                                           - dz_prev * w[i - 1, d]) / prod
                w[i, 0] = -prod_prev * dz_prev * w[i - 1, 0] / prod
            for d in range(top, 0, -1):
                w[j, d] = (dz_last * w[j, d] - d * w[j, d - 1]) / gap
            w[j, 0] = dz_last * w[j, 0] / gap
        prod_prev = prod
    return w


def stencil_start(i: int, ny: int, width: int) -> int:
    """First column of the ``width``-point stencil of row ``i``."""
    return max(0, min(i - width // 2, ny - width))


def diff_bands(y: np.ndarray, p: int):
    """Compact D1 / D2: ``(j0_1, w1[ny, p+1], j0_2, w2[ny, p+2])``."""
    ny = len(y)
    s1, s2 = p + 1, p + 2
    j01 = np.array([stencil_start(i, ny, s1) for i in range(ny)], np.int32)
    j02 = np.array([stencil_start(i, ny, s2) for i in range(ny)], np.int32)
    w1 = np.stack([fornberg_weights(y[i], y[j01[i]:j01[i] + s1], 1)[:, 1]
                   for i in range(ny)])
    w2 = np.stack([fornberg_weights(y[i], y[j02[i]:j02[i] + s2], 2)[:, 2]
                   for i in range(ny)])
    return j01, w1, j02, w2


def build_diff_matrices(y: np.ndarray, p: int):
    """Dense ``(D1, D2)`` from the compact bands."""
    ny = len(y)
    j01, w1, j02, w2 = diff_bands(y, p)
    D1 = np.zeros((ny, ny))
    D2 = np.zeros((ny, ny))
    for i in range(ny):
        D1[i, j01[i]:j01[i] + p + 1] = w1[i]
        D2[i, j02[i]:j02[i] + p + 2] = w2[i]
    return D1, D2


def cgl_grid(ny: int) -> np.ndarray:
    """Chebyshev-Gauss-Lobatto points ``y_j = -cos(j pi/(ny-1))`` on [-1, 1]."""
    return -np.cos(np.arange(ny, dtype=np.float64) * np.pi / (ny - 1))
