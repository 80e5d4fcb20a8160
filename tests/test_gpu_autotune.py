"""Pass variants and the autotuner: every kernel variant of every pass (and
each form of the Couette IMM) gives the default's result to rounding, the
autotuner keeps one of them per pass, and FP32 forms stay on the two-stage
passes."""

from math import pi

import pytest

pytestmark = pytest.mark.gpu


def rel(a, b):
    import torch

    return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))


def periodic(n, fp64=True):
    import torch

    from dnsjax_b200 import initial
    from dnsjax_b200.flows.monochromatic import TriplyPeriodicFlow
    from dnsjax_b200.parameters import Parameters

    p = Parameters(phys=dict(system="kolmogorov", re=40.0), geo=dict(lx=2 * pi, lz=2 * pi),
                   res=dict(nx=n, ny=n, nz=n, double_precision=fp64),
                   step=dict(dt=0.01, corrector_tolerance=1e-10))
    u = initial.periodic_field(n, n, n, 2 * pi, 2 * pi, 2 * pi, 1,
                               initial.kolmogorov_spectrum_cfg0, 1e-2)
    return TriplyPeriodicFlow(p, ly=2 * pi), torch.as_tensor(u, device="cuda")


def couette(n):
    import torch

    from dnsjax_b200 import initial
    from dnsjax_b200.flows.plane_couette import PlaneCouetteFlow
    from dnsjax_b200.parameters import Parameters

    p = Parameters(phys=dict(system="plane-couette", re=400.0), geo=dict(lx=2 * pi, lz=pi),
                   res=dict(nx=n, ny=n + 1, nz=n, fd_order=4),
                   step=dict(dt=0.02, corrector_tolerance=1e-10, max_corrector_iterations=60))
    u = initial.couette_field(n, n + 1, n, 2 * pi, pi, 4, 2, 8.0, 1e-3)
    return PlaneCouetteFlow(p), torch.as_tensor(u, device="cuda")


@pytest.mark.parametrize("var", [[1, 0, 0, 0, 2], [2, 1, 1, 1, 0], [0, 2, 2, 2, 0],
                                 [0, 0, 0, 0, 1]])
def test_periodic_pass_variants(var):
    f, u = periodic(48)
    ref = f.get_rhs(u)
    f.set_variants(var)
    assert rel(f.get_rhs(u), ref) < 1e-12


@pytest.mark.parametrize("var", [[1, 1, 1, 0], [2, 2, 2, 0], [0, 0, 0, 1], [0, 0, 0, 2]])
def test_couette_variants(var):
    f, u = couette(32)
    r_ref = f.get_rhs(u)
    i_ref = f.imm_iteration(u, u, r_ref, r_ref)
    f.set_variants(var)
    r = f.get_rhs(u)
    assert rel(r, r_ref) < 1e-12
    assert rel(f.imm_iteration(u, u, r, r), i_ref) < 1e-12


def test_autotune_choices_and_results():
    from dnsjax_b200 import driver

    f, u = periodic(48)
    ref = f.get_rhs(u)
    t = f.autotune(u, reps=3)
    assert len(t["variants"]) == 5 and all(v in (0, 1, 2) for v in t["variants"])
    for k, v in enumerate(t["variants"]):
        # the fastest, or the default when none is 5% faster than it
        fastest = min(x for x in t["ms"][k] if x >= 0)
        assert t["ms"][k][v] == fastest or (v == 0 and fastest > 0.95 * t["ms"][k][0])
    assert rel(f.get_rhs(u), ref) < 1e-12

    c, uc = couette(32)
    plain = driver.run(c, uc.clone(), 3)
    tc = c.autotune(uc, reps=3)
    assert len(tc["variants"]) == 4 and all(v in (0, 1, 2) for v in tc["variants"])
    tuned = driver.run(c, uc.clone(), 3)
    assert tuned.converged and rel(tuned.state, plain.state) < 1e-10


def test_autotune_fp32_keeps_two_stage_passes():
    from dnsjax_b200 import _lib

    f, u = periodic(48, fp64=False)
    assert f.autotune(u, reps=2)["variants"] == [0, 0, 0, 0, 0]
    with pytest.raises(_lib.DnsbError):
        f.set_variants([0, 1, 1, 1, 0])
