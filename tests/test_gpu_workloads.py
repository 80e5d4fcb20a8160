"""CUDA path against the oracle at the benchmark workloads' sizes.

* Kolmogorov 32^3 (2 pi box, Re 40, dt 0.01, tol 1e-10): 100 steps; every
  velocity component within 1e-10 relative L2 of the FP64 oracle.
* Plane Couette 64x65x64 (p = 4, Re 400, dt 0.02): one full step of the
  reference loop (10 corrector iterations) against the oracle.
* Plane Couette 128x129x128 (p = 6, Re 1000, dt 0.01) and Kolmogorov 128^3:
  single RHS / predictor / corrector calls against the oracle, plus
  size-independent properties (transform round trip, no-slip walls and zero
  wall divergence after the influence-matrix solve).
* The RHS at the other compiled padded lengths (72 and 96: 48^3 and 64^3
  grids) for both flows against the oracle, and the FP32 RHS against the
  FP64 one at padded length 72.
"""

from math import pi

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def dev(a):
    import torch

    return torch.as_tensor(np.ascontiguousarray(a), device="cuda")


def host(t):
    return t.detach().cpu().numpy()


def kolmogorov(n, re, dt, ly=2 * pi, lx=2 * pi, lz=2 * pi, tol=1e-10):
    from dnsjax_b200.flows.monochromatic import TriplyPeriodicFlow
    from dnsjax_b200.parameters import Parameters
    from oracle.config import Config
    from oracle.periodic import PeriodicSetup

    p = Parameters(phys=dict(system="kolmogorov", re=re),
                   geo=dict(lx=lx, lz=lz), res=dict(nx=n, ny=n, nz=n),
                   step=dict(dt=dt, corrector_tolerance=tol))
    cfg = Config(system="kolmogorov", nx=n, ny=n, nz=n, lx=lx, ly=ly, lz=lz,
                 re=re, dt=dt, corrector_tolerance=tol)
    return TriplyPeriodicFlow(p, ly=ly), PeriodicSetup(cfg)


def couette(nx, ny, nz, p_ord, re, dt, tol=1e-10, max_iter=10):
    from dnsjax_b200.flows.plane_couette import PlaneCouetteFlow
    from dnsjax_b200.parameters import Parameters
    from oracle.config import Config
    from oracle.couette import CouetteSetup

    p = Parameters(phys=dict(system="plane-couette", re=re),
                   geo=dict(lx=2 * pi, lz=pi),
                   res=dict(nx=nx, ny=ny, nz=nz, fd_order=p_ord),
                   step=dict(dt=dt, corrector_tolerance=tol,
                             max_corrector_iterations=max_iter))
    flow = PlaneCouetteFlow(p)
    imm = {k: host(v) for k, v in flow.imm.items()}
    imm["D1"], imm["D2"] = flow.D1, flow.D2
    cfg = Config(system="plane-couette", nx=nx, ny=ny, nz=nz, lx=2 * pi,
                 lz=pi, re=re, dt=dt, corrector_tolerance=tol,
                 max_corrector_iterations=max_iter, fd_order=p_ord)
    return flow, CouetteSetup(cfg, imm=imm)


def test_kolmogorov_32_100_steps():
    from dnsjax_b200 import driver, initial
    from oracle.stepper import run

    flow, orc = kolmogorov(32, 40.0, 0.01)
    u0 = initial.periodic_field(32, 32, 32, 2 * pi, 2 * pi, 2 * pi, 0,
                                initial.kolmogorov_spectrum_cfg0, 1e-2)
    res = driver.run(flow, dev(u0), 100)
    ref = run(orc, u0, 100)
    assert res.steps == ref.steps == 100
    assert res.corrector_iterations == ref.corrector_iterations
    got = host(res.state)
    for c in range(3):
        assert rel_l2(got[c], ref.state[c]) <= 1e-10, c


def test_couette_64_one_step():
    from dnsjax_b200 import driver, initial
    from oracle.stepper import run

    flow, orc = couette(64, 65, 64, 4, 400.0, 0.02)
    u0 = initial.couette_field(64, 65, 64, 2 * pi, pi, 4, 1, 8.0, 1e-3)
    res = driver.run(flow, dev(u0), 2)
    ref = run(orc, u0, 2)
    assert res.corrector_iterations == ref.corrector_iterations
    got = host(res.state)
    for c in range(3):
        assert rel_l2(got[c], ref.state[c]) <= 1e-10, c
    assert abs(res.errors[-1] - ref.errors[-1]) <= 1e-6 * ref.errors[-1]


def test_couette_tall_wall_normal_grid():
    """ny = 193 is beyond the batched IMM's wall-normal limit (160), so the
    one-kernel IMM runs, and nx = nz = 16 (padded 24) takes the
    runtime-planned passes: two steps against the oracle."""
    from dnsjax_b200 import driver, initial
    from oracle.stepper import run

    flow, orc = couette(16, 193, 16, 4, 400.0, 0.01, max_iter=60)
    u0 = initial.couette_field(16, 193, 16, 2 * pi, pi, 4, 3, 4.0, 1e-3)
    res = driver.run(flow, dev(u0), 2)
    ref = run(orc, u0, 2)
    assert res.corrector_iterations == ref.corrector_iterations
    got = host(res.state)
    for c in range(3):
        assert rel_l2(got[c], ref.state[c]) <= 1e-10, c


@pytest.fixture(scope="module")
def couette128():
    from dnsjax_b200 import initial

    flow, orc = couette(128, 129, 128, 6, 1000.0, 0.01)
    u0 = initial.couette_field(128, 129, 128, 2 * pi, pi, 6, 4, 32.0, 5e-2)
    return flow, orc, u0


def test_couette_128_calls(couette128):
    flow, orc, u0 = couette128
    r0 = orc.get_rhs(u0)
    g0 = flow.get_rhs(dev(u0))
    assert rel_l2(host(g0), r0) < 1e-12
    p0 = orc.predict(u0, r0)
    gp = flow.predict(dev(u0), dev(r0))
    assert rel_l2(host(gp), p0) < 1e-12
    r1 = orc.get_rhs(p0)
    new, corr = orc.correct(u0, p0, r0, r1)
    gn, gc = flow.correct(dev(u0), dev(p0), dev(r0), dev(r1))
    assert rel_l2(host(gn), new) < 1e-12
    # the correction is the difference of two O(1) states: its relative error
    # is the states' (1e-12) scaled by |new| / |correction|
    amp = np.linalg.norm(new) / np.linalg.norm(corr)
    assert rel_l2(host(gc), corr) < 1e-12 * amp
    assert abs(float(flow.norm(gc).item()) - orc.norm(corr)) < 1e-12 * amp * orc.norm(corr)


def test_couette_128_properties(couette128):
    flow, orc, u0 = couette128
    u = dev(u0)
    # transform round trip
    assert rel_l2(host(flow.phys_to_spec(flow.spec_to_phys(u))), u0) < 1e-13
    # IMM output: no-slip walls, zero wall divergence D1 v (top wall always,
    # bottom wall off the k^2 = 0 mode)
    r = flow.get_rhs(u)
    new = host(flow.predict(u, r))
    vmax = np.abs(new).max()
    assert np.abs(new[..., 0]).max() < 1e-14 * vmax
    assert np.abs(new[..., -1]).max() < 1e-14 * vmax
    dv = np.einsum("j,zxj->zx", flow.D1[0], new[1])
    dt_ = np.einsum("j,zxj->zx", flow.D1[-1], new[1])
    scale = np.abs(new[1]).max() * np.abs(flow.D1[0]).max()
    assert np.abs(dt_).max() < 1e-10 * scale
    dv[0, 0] = 0
    assert np.abs(dv).max() < 1e-10 * scale


def test_kolmogorov_128_rhs():
    from dnsjax_b200 import initial

    flow, orc = kolmogorov(128, 100.0, 0.005)
    u0 = initial.periodic_field(128, 128, 128, 2 * pi, 2 * pi, 2 * pi, 2,
                                initial.kolmogorov_spectrum_k53, 0.5)
    assert rel_l2(host(flow.get_rhs(dev(u0))), orc.get_rhs(u0)) < 1e-12
    phys = flow.spec_to_phys(dev(u0))
    assert rel_l2(host(flow.phys_to_spec(phys)), u0) < 1e-13


@pytest.mark.parametrize("n", [48, 64])
def test_kolmogorov_rhs_sizes(n):
    """Padded lengths 72 and 96 (the 48^3 / 64^3 ensemble members)."""
    from dnsjax_b200 import initial

    flow, orc = kolmogorov(n, 60.0, 0.01)
    u0 = initial.periodic_field(n, n, n, 2 * pi, 2 * pi, 2 * pi, n,
                                initial.kolmogorov_spectrum_cfg0, 1e-2)
    assert rel_l2(host(flow.get_rhs(dev(u0))), orc.get_rhs(u0)) < 1e-12


@pytest.mark.parametrize("n", [48, 64])
def test_couette_rhs_sizes(n):
    """Padded lengths 72 and 96 of the two-stage Couette passes (the x pass
    unpacking rows fastest) against the oracle."""
    from dnsjax_b200 import initial

    flow, orc = couette(n, n + 1, n, 4, 400.0, 0.02)
    u0 = initial.couette_field(n, n + 1, n, 2 * pi, pi, 4, n, 8.0, 1e-3)
    assert rel_l2(host(flow.get_rhs(dev(u0))), orc.get_rhs(u0)) < 1e-12


def test_fp32_rhs_48():
    """The FP32 RHS passes at padded length 72 (48^3 grids) against the FP64
    RHS, both flows (the FP32 pass buffers' rounding: ~1e-7 relative)."""
    from dnsjax_b200 import initial

    flow, _ = couette(48, 49, 48, 4, 400.0, 0.02)
    u = dev(initial.couette_field(48, 49, 48, 2 * pi, pi, 4, 5, 8.0, 1e-3))
    r64 = host(flow.get_rhs(u))
    flow.set_rhs_precision(True)
    r32 = host(flow.get_rhs(u))
    assert rel_l2(r32, r64) < 2e-6
    pflow, _ = kolmogorov(48, 60.0, 0.01)
    u = dev(initial.periodic_field(48, 48, 48, 2 * pi, 2 * pi, 2 * pi, 7,
                                   initial.kolmogorov_spectrum_cfg0, 1e-2))
    r64 = host(pflow.get_rhs(u))
    pflow.set_rhs_precision(True)
    r32 = host(pflow.get_rhs(u))
    assert rel_l2(r32, r64) < 2e-6
