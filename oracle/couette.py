"""Plane-Couette flow (FD in y + influence-matrix method), NumPy FP64.

Oracle restatement (test infrastructure only) of ``src/dnsjax/fd.py``,
``src/dnsjax/geometries/cartesian.py`` and
``src/dnsjax/flows/plane_couette.py``.  Spectral layout ``(3, nz-1,
nx//2, ny)`` in ``[kz, kx, y]`` order; physical ``(3, ny, Mz, Mx)``.

The banded solve is vectorised over modes but performs, per mode, exactly
the operations of the reference's ``_banded_solve_device`` scan
(cartesian.py:360-441): row swap by ``ipiv[j]``, ``kl`` L updates, then
back substitution over ``kl + ku`` U rows with the diagonal at row
``kl + ku``.
"""

from __future__ import annotations

import numpy as np
from scipy.linalg.lapack import get_lapack_funcs

from . import parallel

from .config import Config
from .fft import (
    complex_harmonics,
    get_nonlin,
    phys_to_spec_2d,
    real_harmonics,
    spec_to_phys_2d,
)


# -- fd.py ------------------------------------------------------------------
def fornberg_weights(z: float, x: np.ndarray, m: int) -> np.ndarray:
    """fd.py:21-65: Fornberg (1998) finite-difference weights."""
    n = len(x) - 1
    C = np.zeros((n + 1, m + 1))
    C[0, 0] = 1.0
    c1 = 1.0
    c4 = x[0] - z
    for i in range(1, n + 1):
        mn = min(i, m)
        c2 = 1.0
        c5 = c4
        c4 = x[i] - z
        for j in range(i):
            c3 = x[i] - x[j]
            c2 *= c3
            if j == i - 1:
                for k in range(mn, 0, -1):
                    C[i, k] = c1 * (k * C[i - 1, k - 1] - c5 * C[i - 1, k]) / c2
                C[i, 0] = -c1 * c5 * C[i - 1, 0] / c2
            for k in range(mn, 0, -1):
                C[j, k] = (c4 * C[j, k] - k * C[j, k - 1]) / c3
            C[j, 0] = c4 * C[j, 0] / c3
        c1 = c2
    return C


def build_diff_matrices(y: np.ndarray, p: int):
    """fd.py:68-108: D1 on p+1 points, D2 on p+2 points, one-sided at walls."""
    Ny = len(y)
    s1, s2 = p + 1, p + 2
    h1, h2 = s1 // 2, s2 // 2
    D1 = np.zeros((Ny, Ny))
    D2 = np.zeros((Ny, Ny))
    for i in range(Ny):
        j0 = max(0, min(i - h1, Ny - s1))
        D1[i, j0 : j0 + s1] = fornberg_weights(y[i], y[j0 : j0 + s1], 1)[:, 1]
        j0 = max(0, min(i - h2, Ny - s2))
        D2[i, j0 : j0 + s2] = fornberg_weights(y[i], y[j0 : j0 + s2], 2)[:, 2]
    return D1, D2


def cgl_grid(ny: int) -> np.ndarray:
    """plane_couette.py:73-77: y_j = -cos(j pi / (ny-1))."""
    return -np.cos(np.arange(ny, dtype=float) * np.pi / (ny - 1))


# -- cartesian.py: operators and LU -----------------------------------------
def build_Lk_neumann(k2, D1, D2):
    """cartesian.py:491-526."""
    Ny = D2.shape[0]
    L = D2 - k2 * np.eye(Ny)
    if k2 == 0.0:
        L[0, :] = 0.0
        L[0, 0] = 1.0
        L[-1, :] = D1[-1, :]
    else:
        L[0, :] = D1[0, :]
        L[-1, :] = D1[-1, :]
    return L


def build_Hk_dirichlet(k2, D2, dt, c, nu):
    """cartesian.py:529-572: implicit Hk and explicit Hk_minus."""
    Ny = D2.shape[0]
    Lraw = D2 - k2 * np.eye(Ny)
    Hk = (1.0 / dt) * np.eye(Ny) - c * nu * Lraw
    Hm = (1.0 / dt) * np.eye(Ny) + (1.0 - c) * nu * Lraw
    for H in (Hk, Hm):
        H[0, :] = 0.0
        H[0, 0] = 1.0
        H[-1, :] = 0.0
        H[-1, -1] = 1.0
    return Hk, Hm


def pack_banded(A, kl, ku):
    """cartesian.py:291-320: LAPACK ab packing, A[i,j] at ab[kl+ku+i-j, j]."""
    Ny = A.shape[0]
    ab = np.zeros((2 * kl + ku + 1, Ny), dtype=A.dtype)
    for j in range(Ny):
        for i in range(max(0, j - ku), min(Ny - 1, j + kl) + 1):
            ab[kl + ku + i - j, j] = A[i, j]
    return ab


def banded_lu(A, kl, ku):
    """cartesian.py:323-357: LAPACK dgbtrf; SciPy returns 0-based pivots."""
    ab = pack_banded(A, kl, ku)
    (gbtrf,) = get_lapack_funcs(("gbtrf",), (ab,))
    lu, piv, info = gbtrf(ab, kl, ku, overwrite_ab=True)
    if info != 0:
        raise ValueError(f"dgbtrf failed with info={info}")
    return lu, piv.astype(np.int32)


def banded_solve(ab, ipiv, b, kl, ku):
    """cartesian.py:360-441 (dgbtrs 'N'), vectorised over leading axes.

    ``ab``: (..., 2kl+ku+1, Ny); ``ipiv``: (..., Ny); ``b``: (..., Ny) real.
    With oracle.parallel threads, the modes of the first leading axis are
    split over them.
    """
    ab, ipiv, b = np.asarray(ab), np.asarray(ipiv), np.asarray(b)
    if ab.ndim >= 3 and ab.shape[:-2] == ipiv.shape[:-1] == b.shape[:-1]:
        return parallel.split(lambda a_, p_, b_: _banded_solve_serial(a_, p_, b_, kl, ku),
                              (ab, ipiv, b), 0, n=parallel.SOLVE_THREADS_MAX)
    return _banded_solve_serial(ab, ipiv, b, kl, ku)


def _banded_solve_serial(ab, ipiv, b, kl, ku):
    ab = np.asarray(ab)
    Ny = ab.shape[-1]
    lead = ab.shape[:-2]
    nm = int(np.prod(lead)) if lead else 1
    A = ab.reshape(nm, ab.shape[-2], Ny)
    P = np.asarray(ipiv).reshape(nm, Ny)
    x = np.array(b, dtype=float).reshape(nm, Ny).copy()
    kuu = kl + ku
    xp = np.zeros((nm, Ny + kl))
    xp[:, :Ny] = x
    rows = np.arange(nm)
    for j in range(Ny - 1):
        pj = P[:, j]
        bj = xp[rows, j].copy()
        bpj = xp[rows, pj].copy()
        xp[rows, j] = bpj
        xp[rows, pj] = bj
        lams = A[:, kl + ku + 1 : kl + ku + 1 + kl, j]
        xp[:, j + 1 : j + 1 + kl] = xp[:, j + 1 : j + 1 + kl] - lams * bpj[:, None]
    x = xp[:, :Ny]
    xb = np.zeros((nm, Ny + kuu))
    xb[:, kuu:] = x
    for jr in range(Ny):
        j = Ny - 1 - jr
        jp = j + kuu
        xj = xb[:, jp] / A[:, kl + ku, j]
        xb[:, jp] = xj
        ups = A[:, 0:kuu, j]
        xb[:, jp - kuu : jp] = xb[:, jp - kuu : jp] - ups * xj[:, None]
    return xb[:, kuu:].reshape(lead + (Ny,))


def banded_solve_complex(ab, ipiv, rhs, kl, ku):
    """cartesian.py:444-488: complex RHS split into two real solves."""
    if np.iscomplexobj(rhs):
        xr = banded_solve(ab, ipiv, rhs.real, kl, ku)
        xi = banded_solve(ab, ipiv, rhs.imag, kl, ku)
        return xr + 1j * xi
    return banded_solve(ab, ipiv, rhs, kl, ku)


def precompute_imm(y, kx_vals, kz_vals, p, dt, c, nu, D1=None, D2=None):
    """cartesian.py:575-801 (banded backend)."""
    Ny, Nkz, Nkx = len(y), len(kz_vals), len(kx_vals)
    if D1 is None or D2 is None:
        D1, D2 = build_diff_matrices(y, p)
    kl = ku = p
    rows = 3 * p + 1
    out = {k: np.zeros((Nkz, Nkx, Ny)) for k in ("p1", "p2", "v1", "v2", "q1", "q2")}
    out["M_inv"] = np.zeros((Nkz, Nkx, 2, 2))
    out["Lk_ab"] = np.zeros((Nkz, Nkx, rows, Ny))
    out["Hk_ab"] = np.zeros((Nkz, Nkx, rows, Ny))
    out["Lk_piv"] = np.zeros((Nkz, Nkx, Ny), dtype=np.int32)
    out["Hk_piv"] = np.zeros((Nkz, Nkx, Ny), dtype=np.int32)
    e1 = np.zeros(Ny)
    e1[0] = 1.0
    e2 = np.zeros(Ny)
    e2[-1] = 1.0
    for iz, kz in enumerate(kz_vals):
        for ix, kx in enumerate(kx_vals):
            k2 = float(kx**2 + kz**2)
            Lk = build_Lk_neumann(k2, D1, D2)
            Hk, _ = build_Hk_dirichlet(k2, D2, dt, c, nu)
            p1 = np.linalg.solve(Lk, e1)
            p2 = np.linalg.solve(Lk, e2)
            r1 = -D1 @ p1
            r2 = -D1 @ p2
            r1[0] = r1[-1] = 0.0
            r2[0] = r2[-1] = 0.0
            v1 = np.linalg.solve(Hk, r1)
            v2 = np.linalg.solve(Hk, r2)
            qr1 = p1.copy()
            qr2 = p2.copy()
            qr1[0] = qr1[-1] = 0.0
            qr2[0] = qr2[-1] = 0.0
            q1 = np.linalg.solve(Hk, qr1)
            q2 = np.linalg.solve(Hk, qr2)
            M = np.array(
                [[D1[0] @ v1, D1[0] @ v2], [D1[-1] @ v1, D1[-1] @ v2]]
            )
            if k2 == 0.0:
                Minv = np.array([[0.0, 0.0], [0.0, 1.0 / M[1, 1]]])
            else:
                Minv = np.linalg.inv(M)
            for k, v in (("p1", p1), ("p2", p2), ("v1", v1), ("v2", v2),
                         ("q1", q1), ("q2", q2)):
                out[k][iz, ix] = v
            out["M_inv"][iz, ix] = Minv
            out["Lk_ab"][iz, ix], out["Lk_piv"][iz, ix] = banded_lu(Lk, kl, ku)
            out["Hk_ab"][iz, ix], out["Hk_piv"][iz, ix] = banded_lu(Hk, kl, ku)
    out["D1"], out["D2"] = D1, D2
    return out


def simpson_weights_apply(f: np.ndarray, ys: np.ndarray) -> float:
    """cartesian.py:106-140: non-uniform composite Simpson (odd Ny)."""
    if len(ys) % 2 == 0:
        raise ValueError("Simpson needs an odd number of points")
    h = np.diff(ys)
    h0, h1 = h[:-1:2], h[1::2]
    y0, y1, y2 = f[:-2:2], f[1:-1:2], f[2::2]
    hsum, hprod, r = h0 + h1, h0 * h1, h0 / h1
    panels = (hsum / 6) * (y0 * (2 - 1 / r) + y1 * (hsum**2 / hprod)
                           + y2 * (2 - r))
    return float(np.sum(panels))


class CouetteSetup:
    """cartesian.py:17-69 (Fourier) + plane_couette.py:35-222 (flow data)."""

    def __init__(self, cfg: Config, imm: dict | None = None) -> None:
        self.cfg = cfg
        p = cfg.fd_order
        self.kl = self.ku = p
        kxg = real_harmonics(cfg.nx) * 2 * np.pi / cfg.lx
        kzg = complex_harmonics(cfg.nz) * 2 * np.pi / cfg.lz
        self.kx_global, self.kz_global = kxg, kzg
        self.kx = kxg.reshape(1, -1, 1)
        self.kz = kzg.reshape(-1, 1, 1)
        self.k_metric = np.where(self.kx == 0, 1, 2)
        self.k2 = self.kx**2 + self.kz**2
        self.k2_is_zero = self.k2 == 0.0
        self.ys = cgl_grid(cfg.ny)
        ny = cfg.ny
        U = np.zeros((3, ny))
        U[0] = self.ys
        cU = np.zeros((3, ny))
        cU[2] = -1.0
        nU = np.zeros((3, ny))
        nU[1] = self.ys * 1.0
        self.base_flow = U[:, :, None, None]
        self.curl_base_flow = cU[:, :, None, None]
        self.nonlin_base_flow = nU[:, :, None, None]
        self.nu = 1.0 / cfg.re
        if imm is None:
            imm = precompute_imm(self.ys, kxg, kzg, p, cfg.dt,
                                 cfg.implicitness, self.nu)
        self.imm = imm
        self.D1, self.D2 = imm["D1"], imm["D2"]
        self.D1_bnd = self.D1[[0, -1], :]

    def curl(self, s):
        """plane_couette.py:251-271: D1 in y, i k in x and z."""
        u, v, w = s
        dy_u = parallel.einsum_y(self.D1, u)
        dy_w = parallel.einsum_y(self.D1, w)
        kx, kz = self.kx, self.kz
        return np.array(
            [dy_w - 1j * kz * v, 1j * kz * u - 1j * kx * w, 1j * kx * v - dy_u]
        )

    def get_rhs(self, state):
        """plane_couette.py:274-289 (no projection)."""
        cfg = self.cfg
        return get_nonlin(
            state,
            self.base_flow,
            self.curl_base_flow,
            self.nonlin_base_flow,
            lambda v: spec_to_phys_2d(v, cfg),
            lambda v: phys_to_spec_2d(v, cfg),
            self.curl,
        )

    def lk_matvec(self, u):
        """plane_couette.py:299-338."""
        D2u = parallel.einsum_y(self.D2, u)
        out = D2u - self.k2 * u
        bot_n = np.einsum("j,zxj->zx", self.D1_bnd[0], u)
        bot = np.where(self.k2_is_zero[..., 0], u[..., 0], bot_n)
        top = np.einsum("j,zxj->zx", self.D1_bnd[-1], u)
        out = out.copy()
        out[..., 0] = bot
        out[..., -1] = top
        return out

    def hk_minus_matvec(self, u):
        """plane_couette.py:341-373."""
        c, dt, nu = self.cfg.implicitness, self.cfg.dt, self.nu
        D2u = parallel.einsum_y(self.D2, u)
        out = (1.0 / dt) * u + (1.0 - c) * nu * (D2u - self.k2 * u)
        out = out.copy()
        out[..., 0] = u[..., 0]
        out[..., -1] = u[..., -1]
        return out

    def imm_iteration(self, vel_n, vel_j, nl_n, nl_j):
        """plane_couette.py:376-504: six-stage Kleiser-Schumann IMM."""
        c, dt, nu = self.cfg.implicitness, self.cfg.dt, self.nu
        kx, kz = self.kx, self.kz
        imm, kl, ku = self.imm, self.kl, self.ku
        u_n, v_n, w_n = vel_n
        Nu_n, Nv_n, Nw_n = nl_n
        Nu_j, Nv_j, Nw_j = nl_j
        D1 = self.D1
        dy_v_n = parallel.einsum_y(D1, v_n)
        d_hat = 1j * kx * u_n + dy_v_n + 1j * kz * w_n
        div_Nj = 1j * kx * Nu_j + parallel.einsum_y(D1, Nv_j) + 1j * kz * Nw_j
        div_Nn = 1j * kx * Nu_n + parallel.einsum_y(D1, Nv_n) + 1j * kz * Nw_n
        Lk_d = self.lk_matvec(d_hat)
        f_hat = d_hat / dt + c * div_Nj + (1 - c) * div_Nn + (1 - c) * nu * Lk_d
        f_hat = f_hat.copy()
        f_hat[..., 0] = 0.0
        f_hat[..., -1] = 0.0
        pP = banded_solve_complex(imm["Lk_ab"], imm["Lk_piv"], f_hat, kl, ku)
        dx_p = 1j * kx * pP
        dy_p = parallel.einsum_y(D1, pP)
        dz_p = 1j * kz * pP
        Ru = self.hk_minus_matvec(u_n) - dx_p + c * Nu_j + (1 - c) * Nu_n
        Rv = self.hk_minus_matvec(v_n) - dy_p + c * Nv_j + (1 - c) * Nv_n
        Rw = self.hk_minus_matvec(w_n) - dz_p + c * Nw_j + (1 - c) * Nw_n
        for R in (Ru, Rv, Rw):
            R[..., 0] = 0.0
            R[..., -1] = 0.0
        u_arb = banded_solve_complex(imm["Hk_ab"], imm["Hk_piv"], Ru, kl, ku)
        v_arb = banded_solve_complex(imm["Hk_ab"], imm["Hk_piv"], Rv, kl, ku)
        w_arb = banded_solve_complex(imm["Hk_ab"], imm["Hk_piv"], Rw, kl, ku)
        d_wall = np.einsum("bj,zxj->zxb", self.D1_bnd, v_arb)
        d_wall[..., 0] = np.where(self.k2_is_zero[..., 0], 0.0, d_wall[..., 0])
        alpha = -np.einsum("zxab,zxb->zxa", imm["M_inv"], d_wall)
        a1 = alpha[..., 0][..., None]
        a2 = alpha[..., 1][..., None]
        v_new = v_arb + a1 * imm["v1"] + a2 * imm["v2"]
        q_new = a1 * imm["q1"] + a2 * imm["q2"]
        u_new = u_arb - 1j * kx * q_new
        w_new = w_arb - 1j * kz * q_new
        new = np.array([u_new, v_new, w_new])
        return new, new - vel_j

    def predict(self, state, rhs):
        """plane_couette.py:507-519."""
        new, _ = self.imm_iteration(state, state, rhs, rhs)
        return new

    def correct(self, state_prev, prediction, rhs_prev, rhs_next):
        """plane_couette.py:522-540."""
        return self.imm_iteration(state_prev, prediction, rhs_prev, rhs_next)

    def norm2(self, v):
        """cartesian.py:72-103: modes summed, then Simpson in y, / ly."""
        prof = np.sum((np.conj(v) * self.k_metric * v).real, axis=(0, 1, 2))
        return simpson_weights_apply(prof, self.ys) / self.cfg.ly

    def norm(self, v):
        return float(np.sqrt(self.norm2(v)))

    def correct_velocity(self, state, divergence=True):
        """plane_couette.py:575-582: identity."""
        return state

    def stats(self, state) -> dict:
        """plane_couette.py:591-613: E' only."""
        return {"E'": self.norm2(state) / 2}
