"""The mixed forms (res.double_precision = False): for plane Couette the RHS
transforms and rotational product in FP32, the state, the influence-matrix
iteration (banded LU substitutions, 2x2 solve) and every norm in FP64.

* The FP32 RHS at 128x129x128 against the FP64 oracle: relative L2 per
  component below 2e-6, and not bit-equal to the FP64 path (so the FP32
  kernels are the ones that ran).
* Sizes the FP32 passes do not cover are refused.
* Plane Couette 64x65x64 (p = 4, Re 400, dt 0.02), 20 steps of the reference
  loop from the same seeded field, plain at tolerance 1e-10 and mixed at
  1e-8: the FP32 rounding of the RHS puts a floor under the correction norm
  (about 3e-10 here, about 3e-6 at 128x129x128), so the mixed form is run
  to a tolerance it can reach; the kinetic energy agrees to 1e-6 relative,
  the field to 1e-5 relative L2.
* The periodic flows (Kolmogorov): the same checks for the FP32 y, z and x
  passes, the curl and projection staying FP64, with the dissipation
  compared too.
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


def couette_params(nx, ny, nz, p_ord, re, dt, fp64, tol=1e-10, max_iter=60):
    # corrector tolerance: 1e-10 plain; the caller passes a reachable one for
    # the mixed form
    from dnsjax_b200.parameters import Parameters

    return Parameters(phys=dict(system="plane-couette", re=re),
                      geo=dict(lx=2 * pi, lz=pi),
                      res=dict(nx=nx, ny=ny, nz=nz, fd_order=p_ord,
                               double_precision=fp64),
                      step=dict(dt=dt, corrector_tolerance=tol,
                                max_corrector_iterations=max_iter))


def test_couette_fp32_rhs_128():
    from dnsjax_b200 import initial
    from dnsjax_b200.flows.plane_couette import PlaneCouetteFlow
    from oracle.config import Config
    from oracle.couette import CouetteSetup

    flow = PlaneCouetteFlow(couette_params(128, 129, 128, 6, 1000.0, 0.01, False))
    assert flow.rhs_fp32
    imm = {k: host(v) for k, v in flow.imm.items()}
    imm["D1"], imm["D2"] = flow.D1, flow.D2
    orc = CouetteSetup(Config(system="plane-couette", nx=128, ny=129, nz=128,
                              lx=2 * pi, lz=pi, re=1000.0, dt=0.01, fd_order=6),
                       imm=imm)
    u0 = initial.couette_field(128, 129, 128, 2 * pi, pi, 6, 4, 32.0, 5e-2)
    ref = orc.get_rhs(u0)
    got = host(flow.get_rhs(dev(u0)))
    errs = [rel_l2(got[c], ref[c]) for c in range(3)]
    assert max(errs) < 2e-6, errs
    assert max(errs) > 1e-12, errs  # FP32 arithmetic actually ran


def test_couette_fp32_rejects_runtime_sizes():
    from dnsjax_b200 import _lib
    from dnsjax_b200.flows.plane_couette import PlaneCouetteFlow

    # nx = nz = 16 pad to 24: no compile-time FP32 pass for that length
    flow = PlaneCouetteFlow(couette_params(16, 17, 16, 4, 100.0, 0.01, True))
    with pytest.raises(_lib.DnsbError):
        _lib.check(flow._L.dnsb_couette_set_rhs_precision(flow._ctx, 1))


def test_couette_mixed_trajectory_64():
    from dnsjax_b200 import driver, initial
    from dnsjax_b200.flows.plane_couette import PlaneCouetteFlow

    u0 = initial.couette_field(64, 65, 64, 2 * pi, pi, 4, 1, 8.0, 1e-3)
    plain = PlaneCouetteFlow(couette_params(64, 65, 64, 4, 400.0, 0.02, True))
    mixed = PlaneCouetteFlow(couette_params(64, 65, 64, 4, 400.0, 0.02, False, tol=1e-8))
    rp = driver.run(plain, dev(u0), 20)
    rm = driver.run(mixed, dev(u0), 20)
    assert rm.converged and rp.converged and rm.steps == rp.steps == 20
    assert max(rm.errors) <= 1e-8
    up, um = rp.state, rm.state
    ke = lambda f, u: float(f.norm(u).item()) ** 2 / 2  # noqa: E731
    assert abs(ke(mixed, um) - ke(plain, up)) <= 1e-6 * ke(plain, up)
    a, b = host(um), host(up)
    for c in range(3):
        assert rel_l2(a[c], b[c]) <= 1e-5, c


# -- the periodic flows (Kolmogorov) ---------------------------------------------
def kolmogorov_params(n, re, dt, fp64, tol=1e-10, max_iter=60):
    from dnsjax_b200.parameters import Parameters

    return Parameters(phys=dict(system="kolmogorov", re=re),
                      geo=dict(lx=2 * pi, lz=2 * pi),
                      res=dict(nx=n, ny=n, nz=n, double_precision=fp64),
                      step=dict(dt=dt, corrector_tolerance=tol,
                                max_corrector_iterations=max_iter))


def test_periodic_fp32_rhs_128():
    """The FP32 RHS passes at 128^3 (padded 192^3) against the FP64 RHS
    (itself pinned to the oracle by the parity tests): relative L2 per
    component below 2e-6, and not bit-equal."""
    from dnsjax_b200 import initial
    from dnsjax_b200.flows.monochromatic import TriplyPeriodicFlow

    u0 = dev(initial.periodic_field(128, 128, 128, 2 * pi, 2 * pi, 2 * pi, 2,
                                    initial.kolmogorov_spectrum_k53, 0.5))
    f64 = TriplyPeriodicFlow(kolmogorov_params(128, 100.0, 0.005, True), ly=2 * pi)
    f32 = TriplyPeriodicFlow(kolmogorov_params(128, 100.0, 0.005, False), ly=2 * pi)
    assert f32.rhs_fp32 and not f64.rhs_fp32
    ref = host(f64.get_rhs(u0))
    got = host(f32.get_rhs(u0))
    errs = [rel_l2(got[c], ref[c]) for c in range(3)]
    assert max(errs) < 2e-6, errs
    assert max(errs) > 1e-12, errs


def test_periodic_fp32_rejects_runtime_sizes():
    from dnsjax_b200 import _lib
    from dnsjax_b200.flows.monochromatic import TriplyPeriodicFlow

    # n = 16 pads to 24: no compile-time FP32 pass for that length
    flow = TriplyPeriodicFlow(kolmogorov_params(16, 40.0, 0.01, True), ly=2 * pi)
    with pytest.raises(_lib.DnsbError):
        _lib.check(flow._L.dnsb_periodic_set_rhs_precision(flow._ctx, 1))


def test_periodic_mixed_trajectory_64():
    """Kolmogorov 64^3 (padded 96^3), Re 100, dt 0.005, 20 steps: plain at
    tolerance 1e-10, mixed at 1e-8 (a tolerance above its FP32 floor);
    kinetic energy and dissipation within 1e-6 relative, the field within
    1e-5 relative L2."""
    from dnsjax_b200 import driver, initial
    from dnsjax_b200.flows.monochromatic import TriplyPeriodicFlow

    u0 = initial.periodic_field(64, 64, 64, 2 * pi, 2 * pi, 2 * pi, 3,
                                initial.kolmogorov_spectrum_k53, 0.5)
    plain = TriplyPeriodicFlow(kolmogorov_params(64, 100.0, 0.005, True), ly=2 * pi)
    mixed = TriplyPeriodicFlow(kolmogorov_params(64, 100.0, 0.005, False, tol=1e-8),
                               ly=2 * pi)
    rp = driver.run(plain, dev(u0), 20)
    rm = driver.run(mixed, dev(u0), 20)
    assert rp.converged and rm.converged and rp.steps == rm.steps == 20
    sp, sm = plain.get_stats(rp.state), plain.get_stats(rm.state)
    assert abs(sm["E'"] - sp["E'"]) <= 1e-6 * sp["E'"]
    assert abs(sm["D"] - sp["D"]) <= 1e-6 * abs(sp["D"])
    a, b = host(rm.state), host(rp.state)
    for c in range(3):
        assert rel_l2(a[c], b[c]) <= 1e-5, c


def test_periodic_mixed_1000_steps_128():
    """Kolmogorov 128^3 (padded 192^3), Re 100, dt 0.005, k^-5/3 field of
    energy 0.5: 1000 steps of the mixed form (FP32 transforms and product,
    FP64 projection, corrector norm and reductions; tolerance 1e-8, above
    its FP32 floor) against the plain FP64 form (tolerance 1e-10), both as
    step graphs from the same field.  Kinetic energy and dissipation within
    1e-6 relative and the field within 1e-5 relative L2 at steps 100, 500
    and 1000 (measured: 1.5e-8, 6e-9 and 4.3e-7 at step 1000)."""
    import torch

    from dnsjax_b200 import initial
    from dnsjax_b200.flows.monochromatic import TriplyPeriodicFlow

    u0 = dev(initial.periodic_field(128, 128, 128, 2 * pi, 2 * pi, 2 * pi, 2,
                                    initial.kolmogorov_spectrum_k53, 0.5))
    plain = TriplyPeriodicFlow(kolmogorov_params(128, 100.0, 0.005, True), ly=2 * pi)
    mixed = TriplyPeriodicFlow(kolmogorov_params(128, 100.0, 0.005, False, tol=1e-8),
                               ly=2 * pi)
    marks = (100, 500, 1000)

    def run(flow, tol):
        s = u0.clone()
        g = flow.make_step_graph(s, tol=tol, max_iter=10)
        out = {}
        for k in range(1, 1001):
            g.launch()
            _, e = g.status()
            assert e <= tol, (k, e)
            if k in marks:
                out[k] = s.clone()
        g.close()
        return out

    P, M = run(plain, 1e-10), run(mixed, 1e-8)
    for k in marks:
        sp, sm = plain.get_stats(P[k]), plain.get_stats(M[k])
        assert abs(sm["E'"] - sp["E'"]) <= 1e-6 * sp["E'"], k
        assert abs(sm["D"] - sp["D"]) <= 1e-6 * abs(sp["D"]), k
        d = torch.linalg.vector_norm(M[k] - P[k]) / torch.linalg.vector_norm(P[k])
        assert float(d) <= 1e-5, k


@pytest.mark.parametrize("system", ["plane-couette", "kolmogorov"])
def test_compensated_butterflies_lower_the_fp32_error(system):
    """The FP32 RHS passes with compensated (two-sum) butterflies against the
    plain FP32 passes, both against the FP64 RHS at 128^3 (Couette
    128x129x128 p = 6; Kolmogorov 128^3): per component, the compensated
    error is below the plain FP32 error and below 2e-6 relative L2, and the
    FP64 path is unchanged by switching back."""
    import torch

    from dnsjax_b200 import initial

    if system == "plane-couette":
        from dnsjax_b200.flows.plane_couette import PlaneCouetteFlow
        from dnsjax_b200.parameters import Parameters

        p = Parameters(phys=dict(system="plane-couette", re=1000.0), geo=dict(lx=2 * pi, lz=pi),
                       res=dict(nx=128, ny=129, nz=128, fd_order=6), step=dict(dt=0.01))
        flow = PlaneCouetteFlow(p)
        u = dev(initial.couette_field(128, 129, 128, 2 * pi, pi, 6, 4, 32.0, 5e-2))
    else:
        from dnsjax_b200.flows.monochromatic import TriplyPeriodicFlow

        flow = TriplyPeriodicFlow(kolmogorov_params(128, 100.0, 0.005, True), ly=2 * pi)
        u = dev(initial.periodic_field(128, 128, 128, 2 * pi, 2 * pi, 2 * pi, 2,
                                       initial.kolmogorov_spectrum_k53, 0.5))
    ref = flow.get_rhs(u)
    flow.set_rhs_precision(True)
    plain = flow.get_rhs(u)
    flow.set_rhs_precision(True, compensated=True)
    comp = flow.get_rhs(u)
    flow.set_rhs_precision(False)
    assert torch.equal(flow.get_rhs(u), ref)
    errs = []
    for c in range(3):
        ep = float(torch.linalg.vector_norm(plain[c] - ref[c]) / torch.linalg.vector_norm(ref[c]))
        ec = float(torch.linalg.vector_norm(comp[c] - ref[c]) / torch.linalg.vector_norm(ref[c]))
        errs.append((ep, ec))
        assert ec < ep and ec < 2e-6, (c, ep, ec)
    print(system, errs)
