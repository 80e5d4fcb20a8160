"""Host-side setup of dnsjax_b200 against the reference's own arrays.

The golden fixtures carry the reference's D1/D2, IMM arrays and
Crank-Nicolson coefficients; the package recomputes them with its own code.
"""

import numpy as np
import pytest

from conftest import COUETTE_CASES, PERIODIC_CASES, load_golden, rel_l2


@pytest.mark.parametrize("name", COUETTE_CASES)
def test_fd_and_imm_setup(name):
    from dnsjax_b200.fd import build_diff_matrices, cgl_grid
    from dnsjax_b200.geometries.cartesian import Fourier, precompute_imm

    case, g = load_golden(name)
    ys = cgl_grid(case["ny"])
    D1, D2 = build_diff_matrices(ys, case["p"])
    np.testing.assert_array_equal(D1, g["D1"])
    np.testing.assert_array_equal(D2, g["D2"])
    f = Fourier.build(case["nx"], case["nz"], case["lx"], case["lz"])
    imm = precompute_imm(ys, f.kx_global, f.kz_global, case["p"], case["dt"],
                         0.5, 1.0 / case["re"], D1, D2)
    for k in ("Lk_ab", "Hk_ab", "p1", "p2", "v1", "v2", "q1", "q2", "M_inv"):
        scale = max(1.0, float(np.abs(g[k]).max()))
        np.testing.assert_allclose(imm[k], g[k], rtol=1e-11, atol=1e-12 * scale,
                                   err_msg=k)
    np.testing.assert_array_equal(imm["Lk_piv"], g["Lk_piv"])
    np.testing.assert_array_equal(imm["Hk_piv"], g["Hk_piv"])


def test_simpson_weights_match_panels():
    from dnsjax_b200.fd import cgl_grid
    from dnsjax_b200.geometries.cartesian import simpson_weights
    from oracle.couette import simpson_weights_apply

    ys = cgl_grid(33)
    f = np.random.default_rng(3).standard_normal(33)
    assert abs(simpson_weights(ys) @ f - simpson_weights_apply(f, ys)) < 1e-14
    with pytest.raises(ValueError):
        simpson_weights(cgl_grid(32))


@pytest.mark.parametrize("name", PERIODIC_CASES)
def test_periodic_coefficients(name):
    """ldt_1 / ildt_2 from the package's wavenumbers match the reference."""
    from dnsjax_b200.geometries.triply_periodic import Fourier

    case, g = load_golden(name)
    ly = case["ly"] if case["ly"] is not None else 4.0
    f = Fourier.build(case["nx"], case["ny"], case["nz"], case["lx"], ly, case["lz"])
    dt, c, re = case["dt"], 0.5, case["re"]
    l1 = 1 / dt + (1 - c) * f.lapl / re
    l2 = 1 / (1 / dt - c * f.lapl / re)
    l1[0, 0, 0] = 0
    l2[0, 0, 0] = 0
    assert rel_l2(l1, g["ldt_1"]) == 0.0
    assert rel_l2(l2, g["ildt_2"]) == 0.0


def test_initial_fields_are_divergence_free():
    from dnsjax_b200 import initial

    u = initial.periodic_field(16, 16, 16, 2 * np.pi, 2 * np.pi, 2 * np.pi, 0,
                               initial.kolmogorov_spectrum_cfg0, 1e-2)
    kx = np.arange(8).reshape(1, 1, -1)
    q = np.concatenate([np.arange(8), np.arange(-7, 0)])
    div = kx * u[0] + q.reshape(-1, 1, 1) * u[1] + q.reshape(1, -1, 1) * u[2]
    assert np.abs(div).max() < 1e-14
    assert np.all(u[:, 0, 0, 0] == 0)
    # Hermitian kx = 0 plane: u(-ky, -kz, 0) = conj(u(ky, kz, 0))
    m = (15 - np.arange(15)) % 15
    plane = u[:, :, :, 0]
    assert np.abs(plane - np.conj(plane[:, m][:, :, m])).max() < 1e-15
    k = np.arange(8) != 0
    e = np.sum((np.conj(u) * np.where(kx == 0, 1, 2) * u).real) / 2
    assert abs(e - 1e-2) < 1e-15 and k.any()


def test_couette_initial_field():
    from dnsjax_b200 import initial

    u = initial.couette_field(8, 17, 8, 2 * np.pi, np.pi, 4, 5, 8.0, 1e-3)
    assert u.shape == (3, 7, 4, 17)
    assert np.all(u[..., 0] == 0) and np.all(u[..., -1] == 0)
