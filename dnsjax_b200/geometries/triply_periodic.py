"""Triply-periodic wavenumbers (host setup).

Same grids as the reference's ``Fourier`` (src/dnsjax/geometries/
triply_periodic.py:14-75) and harmonics (src/dnsjax/operators.py:18-56):
``kx = 2 pi/lx [0 .. nx/2-1]``, ``ky``/``kz`` in FFT order with the Nyquist
mode omitted, ``k_metric`` 1 on the kx = 0 plane and 2 elsewhere,
``lapl = -|k|^2`` and ``inv_lapl`` = 1/lapl away from the mean mode.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np


def real_harmonics(n: int) -> np.ndarray:
    return np.arange(0, n // 2, dtype=np.int64)


def complex_harmonics(n: int) -> np.ndarray:
    q = (np.arange(n, dtype=np.int64) + n // 2) % n - n // 2
    return np.concatenate([q[: n // 2], q[n // 2 + 1:]])


@dataclass
class Fourier:
    kx: np.ndarray        # (1, 1, nx/2)
    ky: np.ndarray        # (ny-1, 1, 1)
    kz: np.ndarray        # (1, nz-1, 1)
    k_metric: np.ndarray
    lapl: np.ndarray
    inv_lapl: np.ndarray

    @classmethod
    def build(cls, nx, ny, nz, lx, ly, lz) -> "Fourier":
        kx = real_harmonics(nx).reshape(1, 1, -1) * 2 * np.pi / lx
        kz = complex_harmonics(nz).reshape(1, -1, 1) * 2 * np.pi / lz
        ky = complex_harmonics(ny).reshape(-1, 1, 1) * 2 * np.pi / ly
        k_metric = np.where(kx == 0, 1, 2)
        lapl = -(kx**2 + ky**2 + kz**2)
        with np.errstate(divide="ignore"):
            inv_lapl = np.where(lapl < 0, 1 / lapl, 0.0)
        return cls(kx, ky, kz, k_metric, lapl, inv_lapl)
