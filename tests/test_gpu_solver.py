"""GPU banded solve: the reference's known-answer tests through the C ABI.

Same matrices, seeds and tolerances as the reference's
tests/test_banded_solver.py (lines 68-145), with ``PerModeBandedOperator``
backed by ``dnsb_banded_solve``; plus a batch of many modes against the
oracle's dgbtrs restatement.
"""

import numpy as np
import pytest
from numpy.testing import assert_allclose

from oracle import couette as O

pytestmark = pytest.mark.gpu


def _op(ab, ipiv):
    from dnsjax_b200.geometries.cartesian import PerModeBandedOperator

    return PerModeBandedOperator(ab, ipiv)


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
    x = _op(ab[None, None], ipiv[None, None]).solve(b[None, None, :])
    assert_allclose(x.cpu().numpy()[0, 0], np.linalg.solve(A, b), atol=1e-10,
                    rtol=1e-10)


def test_banded_operator_complex_rhs():
    A = _make_random_banded(16, 4, 4, seed=1)
    rng = np.random.default_rng(11)
    b = rng.standard_normal(16) + 1j * rng.standard_normal(16)
    ab, ipiv = O.banded_lu(A, 4, 4)
    x = _op(ab[None, None], ipiv[None, None]).solve(b[None, None, :])
    assert_allclose(x.cpu().numpy()[0, 0], np.linalg.solve(A, b), atol=1e-10,
                    rtol=1e-10)


def test_banded_vs_dense_on_imm_operators():
    y = -np.cos(np.arange(17) * np.pi / 16)
    D1, D2 = O.build_diff_matrices(y, 4)
    rng = np.random.default_rng(20)
    for kz, kx in [(0.0, 0.0), (0.0, 1.7), (2.0, 3.0)]:
        k2 = kx**2 + kz**2
        Lk = O.build_Lk_neumann(k2, D1, D2)
        Hk, _ = O.build_Hk_dirichlet(k2, D2, 0.01, 0.5, 1e-3)
        b = rng.standard_normal(17) + 1j * rng.standard_normal(17)
        for A in (Lk, Hk):
            ab, ipiv = O.banded_lu(A, 4, 4)
            x = _op(ab[None, None], ipiv[None, None]).solve(b[None, None, :])
            assert_allclose(x.cpu().numpy()[0, 0], np.linalg.solve(A, b),
                            atol=1e-9, rtol=1e-9)


def test_many_modes_against_oracle():
    rng = np.random.default_rng(7)
    Ny, kl = 33, 6
    abs_, pivs = [], []
    for m in range(64):
        # no diagonal shift: partial pivoting must swap rows
        A = _make_random_banded(Ny, kl, kl, seed=100 + m) - 10.0 * np.eye(Ny)
        ab, ipiv = O.banded_lu(A, kl, kl)
        abs_.append(ab)
        pivs.append(ipiv)
    ab = np.stack(abs_).reshape(8, 8, 3 * kl + 1, Ny)
    ipiv = np.stack(pivs).reshape(8, 8, Ny)
    assert (ipiv != np.arange(Ny)).any()  # pivoting is exercised
    b = rng.standard_normal((8, 8, Ny)) + 1j * rng.standard_normal((8, 8, Ny))
    x = _op(ab, ipiv).solve(b).cpu().numpy()
    ref = O.banded_solve_complex(ab, ipiv, b, kl, kl)
    assert np.abs(x - ref).max() <= 1e-11 * np.abs(ref).max()
