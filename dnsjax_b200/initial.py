"""Seeded synthetic initial perturbations (host-side input generation).

The reference starts from the laminar state or from a snapshot
(``flows/monochromatic.py:294-314``, ``flows/plane_couette.py:225-248``);
it ships no random initial fields.  These generators build the seeded
inputs the tests and the benchmark feed to both the oracle and the CUDA
path: a random, divergence-free, Hermitian-consistent spectral field with
a prescribed spectrum, scaled to a prescribed perturbation energy.
"""

from __future__ import annotations

import numpy as np

from .fd import build_diff_matrices, cgl_grid


def _harmonics_real(n):
    return np.arange(n // 2)


def _harmonics_complex(n):
    q = (np.arange(n) + n // 2) % n - n // 2
    return np.concatenate([q[: n // 2], q[n // 2 + 1:]])


def _mirror(n):
    """Index of -q for each stored index q of a Nyquist-free complex axis."""
    i = np.arange(n - 1)
    return (n - 1 - i) % (n - 1)


def periodic_field(nx, ny, nz, lx, ly, lz, seed, spectrum, energy):
    """``(3, ny-1, nz-1, nx//2)`` complex128 field.

    Coefficients are complex Gaussians times ``spectrum(|k|)``; the kx=0
    plane is made Hermitian (what a physical-space round trip does), the
    field is projected divergence-free, the mean mode is zeroed and the
    perturbation energy ``sum(conj(u) k_metric u) / 2`` is set to
    ``energy``.
    """
    rng = np.random.default_rng(seed)
    kx = _harmonics_real(nx).reshape(1, 1, -1) * 2 * np.pi / lx
    ky = _harmonics_complex(ny).reshape(-1, 1, 1) * 2 * np.pi / ly
    kz = _harmonics_complex(nz).reshape(1, -1, 1) * 2 * np.pi / lz
    kk = np.sqrt(kx**2 + ky**2 + kz**2)
    shape = (3, ny - 1, nz - 1, nx // 2)
    u = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) / np.sqrt(2)
    with np.errstate(divide="ignore", invalid="ignore"):
        amp = np.where(kk > 0, spectrum(kk), 0.0)
    u = u * amp
    my, mz = _mirror(ny), _mirror(nz)
    plane = u[:, :, :, 0]
    u[:, :, :, 0] = 0.5 * (plane + np.conj(plane[:, my][:, :, mz]))
    k2 = kk**2
    with np.errstate(divide="ignore", invalid="ignore"):
        kdotu = (kx * u[0] + ky * u[1] + kz * u[2]) / np.where(k2 > 0, k2, 1)
    u = u - np.array([kx * kdotu, ky * kdotu, kz * kdotu])
    u[:, 0, 0, 0] = 0
    kmet = np.where(kx == 0, 1, 2)
    e = np.sum((np.conj(u) * kmet * u).real) / 2
    return np.ascontiguousarray(u * np.sqrt(energy / e))


def couette_field(nx, ny, nz, lx, lz, p, seed, kscale, energy):
    """``(3, nz-1, nx//2, ny)`` complex128 field for plane Couette.

    ``u = curl(psi)`` with ``D1`` in y, so the discrete divergence vanishes;
    ``psi`` has random coefficients with amplitude ``exp(-(kx^2+kz^2)/kscale)``
    times ``(1-y^2)^2`` times a random low-order Chebyshev profile.  The
    kx=0 plane is made Hermitian, wall values are zeroed and the Simpson
    energy (``/ ly`` with ``ly = 2``) is set to ``energy``.
    """
    rng = np.random.default_rng(seed)
    y = cgl_grid(ny)
    D1, _ = build_diff_matrices(y, p)
    kx = (_harmonics_real(nx) * 2 * np.pi / lx).reshape(1, -1, 1)
    kz = (_harmonics_complex(nz) * 2 * np.pi / lz).reshape(-1, 1, 1)
    nkz, nkx = nz - 1, nx // 2
    nm = 4
    cheb = np.stack([np.cos(m * np.arccos(np.clip(y, -1, 1))) for m in range(nm)])
    coef = (rng.standard_normal((3, nkz, nkx, nm))
            + 1j * rng.standard_normal((3, nkz, nkx, nm))) / np.sqrt(2)
    env = (1 - y**2) ** 2
    amp = np.exp(-(kx**2 + kz**2) / kscale)
    psi = np.einsum("czxm,my->czxy", coef, cheb) * env * amp
    dpsi = np.einsum("ij,czxj->czxi", D1, psi)
    u = np.array([
        dpsi[2] - 1j * kz * psi[1],
        1j * kz * psi[0] - 1j * kx * psi[2],
        1j * kx * psi[1] - dpsi[0],
    ])
    mz = _mirror(nz)
    plane = u[:, :, 0, :]
    u[:, :, 0, :] = 0.5 * (plane + np.conj(plane[:, mz]))
    u[..., 0] = 0
    u[..., -1] = 0
    prof = np.sum((np.conj(u) * np.where(kx == 0, 1, 2) * u).real, axis=(0, 1, 2))
    e = simpson(prof, y) / 2.0 / 2
    return np.ascontiguousarray(u * np.sqrt(energy / e))


def simpson(f, ys):
    """Composite Simpson on non-uniform panels (odd number of points)."""
    h = np.diff(ys)
    h0, h1 = h[:-1:2], h[1::2]
    r = h0 / h1
    hs = h0 + h1
    return float(np.sum((hs / 6) * (f[:-2:2] * (2 - 1 / r)
                                    + f[1:-1:2] * (hs**2 / (h0 * h1))
                                    + f[2::2] * (2 - r))))


def kolmogorov_spectrum_cfg0(k):
    """Amplitude k^-2 exp(-k^2/16) (32^3 Kolmogorov workload)."""
    return k**-2.0 * np.exp(-k**2 / 16)


def kolmogorov_spectrum_k53(k):
    """Amplitude k^-5/3 exp(-k^2/400) (128^3 Kolmogorov workload)."""
    return k ** (-5.0 / 3.0) * np.exp(-k**2 / 400)
