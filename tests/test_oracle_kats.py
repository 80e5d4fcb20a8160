"""The reference's banded-solver known-answer tests, restated on the oracle.

Same matrices, seeds and tolerances as tests/test_banded_solver.py of the
reference (its lines 55-197): a random banded matrix with a +10 I shift,
complex right-hand sides via the split real/imaginary path, L_k / H_k on a
17-point CGL grid at modes (kz, kx) in {(0,0), (0,1.7), (2,3)} -- including
the k^2 = 0 pin -- against dense solves, and the two matrix-free matvecs
against the dense operators.
"""

import numpy as np
from numpy.testing import assert_allclose

from oracle import couette as O


def _make_random_banded(Ny, kl, ku, seed):
    rng = np.random.default_rng(seed)
    A = np.zeros((Ny, Ny))
    for i in range(Ny):
        lo, hi = max(0, i - kl), min(Ny, i + ku + 1)
        A[i, lo:hi] = rng.standard_normal(hi - lo)
    return A + 10.0 * np.eye(Ny)


def test_banded_solve_random_real():
    A = _make_random_banded(16, 4, 4, seed=0)
    b = np.random.default_rng(10).standard_normal(16)
    ab, ipiv = O.banded_lu(A, 4, 4)
    x = O.banded_solve(ab, ipiv, b, 4, 4)
    assert_allclose(x, np.linalg.solve(A, b), atol=1e-10, rtol=1e-10)


def test_banded_operator_complex_rhs():
    A = _make_random_banded(16, 4, 4, seed=1)
    rng = np.random.default_rng(11)
    b = rng.standard_normal(16) + 1j * rng.standard_normal(16)
    ab, ipiv = O.banded_lu(A, 4, 4)
    x = O.banded_solve_complex(ab[None, None], ipiv[None, None],
                               b[None, None, :], 4, 4)[0, 0]
    assert_allclose(x, np.linalg.solve(A, b), atol=1e-10, rtol=1e-10)


MODES = [(0.0, 0.0), (0.0, 1.7), (2.0, 3.0)]


def _grid(Ny=17, p=4):
    y = -np.cos(np.arange(Ny) * np.pi / (Ny - 1))
    return y, *O.build_diff_matrices(y, p)


def test_banded_vs_dense_on_imm_operators():
    _, D1, D2 = _grid()
    rng = np.random.default_rng(20)
    for kz, kx in MODES:
        k2 = kx**2 + kz**2
        Lk = O.build_Lk_neumann(k2, D1, D2)
        Hk, _ = O.build_Hk_dirichlet(k2, D2, 0.01, 0.5, 1e-3)
        b = rng.standard_normal(17) + 1j * rng.standard_normal(17)
        for A in (Lk, Hk):
            ab, ipiv = O.banded_lu(A, 4, 4)
            x = O.banded_solve_complex(ab, ipiv, b, 4, 4)
            assert_allclose(x, np.linalg.solve(A, b), atol=1e-9, rtol=1e-9)


class _Probe(O.CouetteSetup):
    """Just enough of CouetteSetup to call the two matvecs on one mode."""

    def __init__(self, D1, D2, k2, dt=0.01, c=0.5, nu=1e-3):
        from oracle.config import Config

        self.cfg = Config(system="plane-couette", dt=dt, implicitness=c)
        self.nu = nu
        self.D1, self.D2 = D1, D2
        self.D1_bnd = D1[[0, -1], :]
        self.k2 = np.array([[[k2]]])
        self.k2_is_zero = self.k2 == 0.0


def test_lk_matvec_matches_dense():
    _, D1, D2 = _grid()
    rng = np.random.default_rng(30)
    for kz, kx in MODES:
        k2 = kx**2 + kz**2
        u = rng.standard_normal(17) + 1j * rng.standard_normal(17)
        got = _Probe(D1, D2, k2).lk_matvec(u[None, None, :])[0, 0]
        assert_allclose(got, O.build_Lk_neumann(k2, D1, D2) @ u, atol=1e-10,
                        rtol=1e-10)


def test_hk_minus_matvec_matches_dense():
    _, D1, D2 = _grid()
    rng = np.random.default_rng(40)
    for kz, kx in MODES:
        k2 = kx**2 + kz**2
        _, Hm = O.build_Hk_dirichlet(k2, D2, 0.01, 0.5, 1e-3)
        u = rng.standard_normal(17) + 1j * rng.standard_normal(17)
        got = _Probe(D1, D2, k2).hk_minus_matvec(u[None, None, :])[0, 0]
        assert_allclose(got, Hm @ u, atol=1e-10, rtol=1e-10)
