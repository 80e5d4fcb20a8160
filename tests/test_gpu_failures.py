"""Failure detection on the GPU, with no GPU fault: every failure is made
on the host (a corrupted operator, a wait limit that nothing can meet, a
non-finite field) and read back as a status or an exception.

* A pivot index outside [j, j+kl] in the banded LU factors: the
  standalone solve (``PerModeBandedOperator.solve``,
  geometries/cartesian.py:360-488 of the reference) raises, and binding such
  operators to a plane-Couette context sets the status that
  ``check_status`` raises; the bad pivot is never followed.
* The IMM substitution's shared-memory ring waits are bounded: with a limit
  of zero polls every wait gives up at once; the call sets the status bit,
  drains its copies and returns, the context stays usable, and after the
  status is cleared and the limit restored the next call matches the oracle.
* A non-finite initial field ends the run after its first step, as the
  reference's loop does (``__main__.py:125-129``: it steps while
  last_error < corrector_tolerance), through the host loop and the step
  graph alike.
"""

from math import pi

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _couette(nx=32, ny=33, nz=32, p_ord=4, imm=None, max_iter=60):
    from dnsjax_b200.flows.plane_couette import PlaneCouetteFlow
    from dnsjax_b200.parameters import Parameters

    params = Parameters(phys=dict(system="plane-couette", re=400.0),
                        geo=dict(lx=2 * pi, lz=pi),
                        res=dict(nx=nx, ny=ny, nz=nz, fd_order=p_ord),
                        step=dict(dt=0.02, corrector_tolerance=1e-10,
                                  max_corrector_iterations=max_iter))
    return PlaneCouetteFlow(params, imm=imm)


def test_banded_solve_rejects_out_of_range_pivot():
    import torch

    from dnsjax_b200 import _lib
    from dnsjax_b200.geometries.cartesian import PerModeBandedOperator
    from oracle.couette import banded_lu

    rng = np.random.default_rng(3)
    ny, kl = 17, 4
    abs_, pivs = [], []
    for _ in range(3):
        A = np.diag(rng.uniform(1, 2, ny))
        for d in range(1, kl + 1):
            A += np.diag(rng.standard_normal(ny - d), d) + np.diag(rng.standard_normal(ny - d), -d)
        lu, piv = banded_lu(A, kl, kl)
        abs_.append(lu)
        pivs.append(piv)
    ab = torch.as_tensor(np.stack(abs_), device="cuda")
    piv = np.stack(pivs)
    good = PerModeBandedOperator(ab, torch.as_tensor(piv, device="cuda"))
    b = rng.standard_normal((3, ny))
    x = good.solve(b).cpu().numpy()
    assert np.all(np.isfinite(x))
    bad = piv.copy()
    bad[1, 5] = 5 + kl + 3  # beyond the kl rows below the diagonal
    op = PerModeBandedOperator(ab, torch.as_tensor(bad, device="cuda"))
    with pytest.raises(_lib.DnsbError, match="pivot"):
        op.solve(b)
    bad[1, 5] = 4  # above the diagonal
    op = PerModeBandedOperator(ab, torch.as_tensor(bad, device="cuda"))
    with pytest.raises(_lib.DnsbError, match="pivot"):
        op.solve(b)


def test_couette_context_flags_bad_pivot_at_bind():
    import torch

    from dnsjax_b200 import _lib, initial

    good = _couette()
    good.check_status()
    imm = {k: v.clone() for k, v in good.imm.items()}
    imm["Hk_piv"][2, 3, 7] = 7 + good.p + 2
    flow = _couette(imm=imm)
    with pytest.raises(_lib.DnsbError, match="pivot"):
        flow.check_status()
    # the flagged context still runs (the pivot is not followed): finite output
    u = torch.as_tensor(initial.couette_field(32, 33, 32, 2 * pi, pi, 4, 1, 8.0, 1e-3),
                        device="cuda")
    r = flow.get_rhs(u)
    out = flow.predict(u, r)
    assert bool(torch.isfinite(torch.view_as_real(out)).all())


def test_imm_ring_wait_gives_up_and_recovers():
    import torch

    from dnsjax_b200 import _lib, initial
    from oracle.config import Config
    from oracle.couette import CouetteSetup

    flow = _couette()
    u0 = initial.couette_field(32, 33, 32, 2 * pi, pi, 4, 2, 8.0, 1e-3)
    u = torch.as_tensor(u0, device="cuda")
    r = flow.get_rhs(u)
    flow.check_status()
    flow.set_wait_limit(0)  # every ring wait gives up on its first poll
    flow.predict(u, r)
    with pytest.raises(_lib.DnsbError, match="ring wait timed out"):
        flow.check_status()
    with pytest.raises(_lib.DnsbError):  # sticky until cleared
        flow.check_status()
    flow.clear_status()
    flow.set_wait_limit(1 << 20)
    flow.check_status()
    got = flow.predict(u, r).cpu().numpy()
    flow.check_status()
    imm = {k: v.cpu().numpy() for k, v in flow.imm.items()}
    imm["D1"], imm["D2"] = flow.D1, flow.D2
    orc = CouetteSetup(Config(system="plane-couette", nx=32, ny=33, nz=32, lx=2 * pi, lz=pi,
                              re=400.0, dt=0.02, corrector_tolerance=1e-10, fd_order=4),
                       imm=imm)
    want = orc.predict(u0, orc.get_rhs(u0))
    assert rel_l2(got, want) < 1e-12


@pytest.mark.parametrize("system", ["plane-couette", "kolmogorov"])
def test_non_finite_field_ends_the_run(system):
    import torch

    from dnsjax_b200 import driver, initial

    if system == "plane-couette":
        flow = _couette()
        u0 = initial.couette_field(32, 33, 32, 2 * pi, pi, 4, 1, 8.0, 1e-3)
    else:
        from dnsjax_b200.flows.monochromatic import TriplyPeriodicFlow
        from dnsjax_b200.parameters import Parameters

        p = Parameters(phys=dict(system="kolmogorov", re=40.0), geo=dict(lx=2 * pi, lz=2 * pi),
                       res=dict(nx=16, ny=16, nz=16),
                       step=dict(dt=0.01, corrector_tolerance=1e-10))
        flow = TriplyPeriodicFlow(p, ly=2 * pi)
        u0 = initial.periodic_field(16, 16, 16, 2 * pi, 2 * pi, 2 * pi, 0,
                                    initial.kolmogorov_spectrum_cfg0, 1e-2)
    u0[0, 1, 1, 1] = np.nan
    res = driver.run(flow, torch.as_tensor(u0, device="cuda"), 5)
    assert res.steps == 1 and not res.converged
    assert res.corrector_iterations == [0] and not np.isfinite(res.errors[0])
    # the step graph's device-controlled loop stops on the same condition
    state = torch.as_tensor(u0, device="cuda")
    g = flow.make_step_graph(state, tol=1e-10, max_iter=60)
    g.launch()
    it, err = g.status()
    g.close()
    assert it == 0 and not np.isfinite(err)
