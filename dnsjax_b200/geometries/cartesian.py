"""Cartesian wall-bounded geometry: wavenumbers, IMM operators, banded solve.

Host-side setup mirrors the reference (src/dnsjax/geometries/cartesian.py):

* ``Fourier`` -- ``kx``, ``kz``, ``k_metric``, ``k2`` (cartesian.py:17-69);
* ``precompute_imm`` -- per-(kz, kx) influence-matrix data and LAPACK
  ``gbtrf`` banded LU factors of ``L_k`` (Neumann) and ``H_k`` (Dirichlet)
  in the reference's ``ab`` layout (cartesian.py:491-801), on the host as
  the reference runs it (this version batches the dense homogeneous solves
  across modes);
* ``precompute_imm_gpu`` -- the same arrays computed on the GPU
  (``dnsb_imm_precompute``);
* ``simpson_weights`` -- the non-uniform composite Simpson rule of
  cartesian.py:106-140 as a linear functional.

``PerModeBandedOperator.solve`` (cartesian.py:444-488) runs on the GPU
through ``dnsb_banded_solve``.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
from scipy.linalg.lapack import get_lapack_funcs

from .triply_periodic import complex_harmonics, real_harmonics


@dataclass
class Fourier:
    kx_global: np.ndarray
    kz_global: np.ndarray
    kx: np.ndarray          # (1, nx/2, 1)
    kz: np.ndarray          # (nz-1, 1, 1)
    k_metric: np.ndarray
    k2: np.ndarray
    k2_is_zero: np.ndarray

    @classmethod
    def build(cls, nx, nz, lx, lz) -> "Fourier":
        kxg = real_harmonics(nx) * 2 * np.pi / lx
        kzg = complex_harmonics(nz) * 2 * np.pi / lz
        kx = kxg.reshape(1, -1, 1)
        kz = kzg.reshape(-1, 1, 1)
        k2 = kx**2 + kz**2
        return cls(kxg, kzg, kx, kz, np.where(kx == 0, 1, 2), k2, k2 == 0.0)


def simpson_weights(ys: np.ndarray) -> np.ndarray:
    """W with sum(W * f) = composite Simpson of f on the grid ys (odd n)."""
    n = len(ys)
    if n % 2 == 0:
        raise ValueError("Simpson integration needs an odd number of points")
    W = np.zeros(n)
    for i in range(0, n - 2, 2):
        h0, h1 = ys[i + 1] - ys[i], ys[i + 2] - ys[i + 1]
        hs, hp, r = h0 + h1, h0 * h1, h0 / h1
        W[i] += (hs / 6) * (2 - 1 / r)
        W[i + 1] += (hs / 6) * (hs**2 / hp)
        W[i + 2] += (hs / 6) * (2 - r)
    return W


def _lk_neumann(k2: np.ndarray, D1, D2) -> np.ndarray:
    """Batched L_k = D2 - k2 I with Neumann wall rows; k2 = 0 pins p[0]."""
    ny = D2.shape[0]
    L = D2[None] - k2[:, None, None] * np.eye(ny)[None]
    z = k2 == 0.0
    L[:, 0, :] = D1[0]
    L[z, 0, :] = 0.0
    L[z, 0, 0] = 1.0
    L[:, -1, :] = D1[-1]
    return L


def _hk_dirichlet(k2: np.ndarray, D2, dt, c, nu) -> np.ndarray:
    """Batched implicit H_k = I/dt - c nu (D2 - k2 I), identity wall rows."""
    ny = D2.shape[0]
    eye = np.eye(ny)
    Lraw = D2[None] - k2[:, None, None] * eye[None]
    H = (1.0 / dt) * eye[None] - c * nu * Lraw
    H[:, 0, :] = 0.0
    H[:, 0, 0] = 1.0
    H[:, -1, :] = 0.0
    H[:, -1, -1] = 1.0
    return H


def pack_banded(A: np.ndarray, kl: int, ku: int) -> np.ndarray:
    """LAPACK ab packing of (..., n, n): A[i, j] -> ab[kl+ku+i-j, j]."""
    n = A.shape[-1]
    ab = np.zeros(A.shape[:-2] + (2 * kl + ku + 1, n), dtype=A.dtype)
    for d in range(-ku, kl + 1):  # d = i - j
        j = np.arange(max(0, -d), min(n, n - d))
        ab[..., kl + ku + d, j] = A[..., j + d, j]
    return ab


def banded_lu(ab: np.ndarray, kl: int, ku: int):
    """LAPACK gbtrf of one packed matrix; 0-based pivots (SciPy)."""
    (gbtrf,) = get_lapack_funcs(("gbtrf",), (ab,))
    lu, piv, info = gbtrf(ab, kl, ku, overwrite_ab=False)
    if info != 0:
        raise ValueError(f"dgbtrf failed with info={info}")
    return lu, piv.astype(np.int32)


def precompute_imm(y, kx_vals, kz_vals, p, dt, c, nu, D1, D2,
                   chunk_modes: int = 1024) -> dict:
    """Influence-matrix data for all (kz, kx) modes (banded backend).

    Returns p1, p2, v1, v2, q1, q2 ``(Nkz, Nkx, Ny)``, M_inv
    ``(Nkz, Nkx, 2, 2)``, Lk_ab / Hk_ab ``(Nkz, Nkx, 3p+1, Ny)`` and
    Lk_piv / Hk_piv ``(Nkz, Nkx, Ny)`` int32, as the reference's
    ``precompute_imm`` does.
    """
    ny, nkz, nkx = len(y), len(kz_vals), len(kx_vals)
    kl = ku = p
    k2_all = (kx_vals[None, :] ** 2 + kz_vals[:, None] ** 2).reshape(-1)
    nm = k2_all.size
    out = {k: np.zeros((nm, ny)) for k in ("p1", "p2", "v1", "v2", "q1", "q2")}
    out["M_inv"] = np.zeros((nm, 2, 2))
    out["Lk_ab"] = np.zeros((nm, 3 * p + 1, ny))
    out["Hk_ab"] = np.zeros((nm, 3 * p + 1, ny))
    out["Lk_piv"] = np.zeros((nm, ny), np.int32)
    out["Hk_piv"] = np.zeros((nm, ny), np.int32)
    E = np.zeros((ny, 2))
    E[0, 0] = 1.0
    E[-1, 1] = 1.0
    for s in range(0, nm, chunk_modes):
        k2 = k2_all[s:s + chunk_modes]
        b = k2.size
        Lk = _lk_neumann(k2, D1, D2)
        Hk = _hk_dirichlet(k2, D2, dt, c, nu)
        P = np.linalg.solve(Lk, np.broadcast_to(E, (b, ny, 2)))
        R = np.concatenate([-(D1 @ P), P], axis=2)  # -D1 p1, -D1 p2, p1, p2
        R[:, 0, :] = 0.0
        R[:, -1, :] = 0.0
        V = np.linalg.solve(Hk, R)
        out["p1"][s:s + b] = P[..., 0]
        out["p2"][s:s + b] = P[..., 1]
        out["v1"][s:s + b] = V[..., 0]
        out["v2"][s:s + b] = V[..., 1]
        out["q1"][s:s + b] = V[..., 2]
        out["q2"][s:s + b] = V[..., 3]
        M = np.empty((b, 2, 2))
        M[:, 0, 0] = V[..., 0] @ D1[0]
        M[:, 0, 1] = V[..., 1] @ D1[0]
        M[:, 1, 0] = V[..., 0] @ D1[-1]
        M[:, 1, 1] = V[..., 1] @ D1[-1]
        Mi = np.zeros((b, 2, 2))
        z = k2 == 0.0
        if np.any(~z):
            Mi[~z] = np.linalg.inv(M[~z])
        Mi[z, 1, 1] = 1.0 / M[z, 1, 1]
        out["M_inv"][s:s + b] = Mi
        Lab = pack_banded(Lk, kl, ku)
        Hab = pack_banded(Hk, kl, ku)
        for i in range(b):
            out["Lk_ab"][s + i], out["Lk_piv"][s + i] = banded_lu(Lab[i], kl, ku)
            out["Hk_ab"][s + i], out["Hk_piv"][s + i] = banded_lu(Hab[i], kl, ku)
    for k, v in out.items():
        out[k] = v.reshape((nkz, nkx) + v.shape[1:])
    out["D1"], out["D2"] = D1, D2
    return out


IMM_KEYS_F64 = ("p1", "p2", "v1", "v2", "q1", "q2", "M_inv", "Lk_ab", "Hk_ab")


def precompute_imm_gpu(kx_vals, kz_vals, p, dt, c, nu, D1, D2) -> dict:
    """``precompute_imm`` on the GPU (``dnsb_imm_precompute``): the same keys
    and shapes as device tensors (cartesian.py:575-801).  The operators are
    built and factored per mode exactly as the reference packs and factors
    them (LAPACK dgbtf2 with partial pivoting); p, v, q are solved with the
    banded factors instead of dense LU, so they agree to rounding.  Raises
    ValueError on a zero pivot, as the reference does for LAPACK info > 0."""
    import torch

    from .. import _lib

    L = _lib.lib()
    ny, nkx, nkz = D1.shape[0], len(kx_vals), len(kz_vals)

    def dev(a):
        return torch.as_tensor(np.ascontiguousarray(a, np.float64), device="cuda")

    d1, d2, kx, kz = dev(D1), dev(D2), dev(kx_vals), dev(kz_vals)
    f64 = dict(dtype=torch.float64, device="cuda")
    out = {k: torch.empty((nkz, nkx, ny), **f64) for k in ("p1", "p2", "v1", "v2", "q1", "q2")}
    out["M_inv"] = torch.empty((nkz, nkx, 2, 2), **f64)
    for k in ("Lk", "Hk"):
        out[k + "_ab"] = torch.empty((nkz, nkx, 3 * p + 1, ny), **f64)
        out[k + "_piv"] = torch.empty((nkz, nkx, ny), dtype=torch.int32, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    ptr = _lib.ptr
    _lib.check(L.dnsb_imm_precompute(
        ptr(d1), ptr(d2), ptr(kx), nkx, ptr(kz), nkz, ny, p, float(dt), float(c), float(nu),
        *[ptr(out[k]) for k in ("p1", "p2", "v1", "v2", "q1", "q2", "M_inv", "Lk_ab",
                                 "Lk_piv", "Hk_ab", "Hk_piv")],
        ptr(info), _lib.stream_handle()))
    bad = int(info.item())
    if bad & 6:
        which = " and ".join(n for b, n in ((2, "L_k"), (4, "H_k")) if bad & b)
        raise ValueError(f"dgbtrf failed: zero pivot in some {which}")
    out["D1"], out["D2"] = D1, D2
    return out


class PerModeBandedOperator:
    """Per-mode LAPACK-``ab`` LU factors on the GPU; ``solve`` runs
    ``dnsb_banded_solve`` (dgbtrs 'N'), complex right-hand sides as two real
    columns (cartesian.py:444-488)."""

    def __init__(self, ab, ipiv):
        import torch

        self.ab = torch.as_tensor(ab, dtype=torch.float64, device="cuda").contiguous()
        self.ipiv = torch.as_tensor(ipiv, dtype=torch.int32, device="cuda").contiguous()
        p3 = self.ab.shape[-2]
        if (p3 - 1) % 3:
            raise ValueError("ab must have 3p+1 rows")
        self.kl = self.ku = (p3 - 1) // 3

    def solve(self, rhs):
        import torch

        from .. import _lib

        L = _lib.lib()
        ny = self.ab.shape[-1]
        nmodes = self.ab.numel() // (self.ab.shape[-2] * ny)
        x = torch.as_tensor(rhs, device="cuda").clone().contiguous()
        if x.is_complex():
            buf = torch.view_as_real(x).contiguous()
            ncols = 2
        else:
            buf = x.to(torch.float64)
            ncols = 1
        status = torch.zeros(1, dtype=torch.int32, device="cuda")
        _lib.check(L.dnsb_banded_solve(
            _lib.ptr(self.ab), _lib.ptr(self.ipiv), _lib.ptr(buf), nmodes, ny,
            self.kl, self.ku, ncols, _lib.ptr(status), _lib.stream_handle()))
        if int(status.item()) != 0:
            raise _lib.DnsbError("pivot index outside [j, j+kl]")
        if ncols == 2:
            return torch.view_as_complex(buf)
        return buf
