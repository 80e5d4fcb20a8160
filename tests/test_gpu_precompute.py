"""Influence-matrix precompute on the GPU (dnsb_imm_precompute) against the
reference's own arrays and the host restatement.

* Golden cases (the reference's precompute_imm, cartesian.py:575-801): the
  factors, homogeneous solutions and M_inv within the tolerances the host
  setup test uses (rtol 1e-11), the pivots equal.
* Plane Couette 64x65x64 (p = 4) and a slice of 128x129x128 (p = 6): the
  same against the host precompute.
* A plane-Couette trajectory with GPU-precomputed operators stays within
  rounding of one with host-precomputed operators.
* A singular L_k (zero derivative matrices) raises ValueError, as the
  reference's gbtrf info check does.
"""

from math import pi

import numpy as np
import pytest

from conftest import COUETTE_CASES, load_golden

pytestmark = pytest.mark.gpu

F64_KEYS = ("Lk_ab", "Hk_ab", "p1", "p2", "v1", "v2", "q1", "q2", "M_inv")


def host(t):
    return t.detach().cpu().numpy()


def assert_imm_close(got, ref):
    for k in F64_KEYS:
        g = host(got[k]) if not isinstance(got[k], np.ndarray) else got[k]
        scale = max(1.0, float(np.abs(ref[k]).max()))
        np.testing.assert_allclose(g, ref[k], rtol=1e-11, atol=1e-12 * scale, err_msg=k)
    for k in ("Lk_piv", "Hk_piv"):
        np.testing.assert_array_equal(host(got[k]), ref[k], err_msg=k)


@pytest.mark.parametrize("name", COUETTE_CASES)
def test_gpu_precompute_matches_reference_arrays(name):
    from dnsjax_b200.fd import build_diff_matrices, cgl_grid
    from dnsjax_b200.geometries.cartesian import Fourier, precompute_imm_gpu

    case, g = load_golden(name)
    ys = cgl_grid(case["ny"])
    D1, D2 = build_diff_matrices(ys, case["p"])
    f = Fourier.build(case["nx"], case["nz"], case["lx"], case["lz"])
    imm = precompute_imm_gpu(f.kx_global, f.kz_global, case["p"], case["dt"], 0.5,
                             1.0 / case["re"], D1, D2)
    assert_imm_close(imm, g)


@pytest.mark.parametrize("n,ny,p,nz_slice", [(64, 65, 4, None), (128, 129, 6, 12)])
def test_gpu_precompute_matches_host(n, ny, p, nz_slice):
    from dnsjax_b200.fd import build_diff_matrices, cgl_grid
    from dnsjax_b200.geometries.cartesian import Fourier, precompute_imm, precompute_imm_gpu

    ys = cgl_grid(ny)
    D1, D2 = build_diff_matrices(ys, p)
    f = Fourier.build(n, n, 2 * pi, pi)
    kz = f.kz_global if nz_slice is None else f.kz_global[::len(f.kz_global) // nz_slice]
    ref = precompute_imm(ys, f.kx_global, kz, p, 0.01, 0.5, 1e-3, D1, D2)
    got = precompute_imm_gpu(f.kx_global, kz, p, 0.01, 0.5, 1e-3, D1, D2)
    assert_imm_close(got, ref)


def test_gpu_precompute_trajectory():
    import torch

    from dnsjax_b200 import driver, initial
    from dnsjax_b200.flows.plane_couette import PlaneCouetteFlow
    from dnsjax_b200.parameters import Parameters

    p = Parameters(phys=dict(system="plane-couette", re=400.0),
                   geo=dict(lx=2 * pi, lz=pi), res=dict(nx=64, ny=65, nz=64, fd_order=4),
                   step=dict(dt=0.02, corrector_tolerance=1e-10, max_corrector_iterations=60))
    u0 = initial.couette_field(64, 65, 64, 2 * pi, pi, 4, 1, 8.0, 1e-3)
    fg = PlaneCouetteFlow(p, precompute="gpu")
    fh = PlaneCouetteFlow(p, precompute="host")
    rg = driver.run(fg, torch.as_tensor(u0, device="cuda"), 5)
    rh = driver.run(fh, torch.as_tensor(u0, device="cuda"), 5)
    assert rg.converged and rh.converged
    d = torch.linalg.vector_norm(rg.state - rh.state) / torch.linalg.vector_norm(rh.state)
    assert float(d) < 1e-12


def test_gpu_precompute_zero_pivot_raises():
    from dnsjax_b200.geometries.cartesian import Fourier, precompute_imm_gpu

    ny = 17
    Z = np.zeros((ny, ny))
    f = Fourier.build(8, 8, 2 * pi, pi)
    with pytest.raises(ValueError, match="L_k"):
        precompute_imm_gpu(f.kx_global, f.kz_global, 4, 0.01, 0.5, 1e-3, Z, Z)
