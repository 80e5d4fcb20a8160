"""CUDA path against the reference's golden vectors (small grids).

Every golden case (tests/golden, produced by the reference's own source)
is replayed through the C ABI: transforms, RHS, predictor, corrector and
its fused norm, divergence correction, stats, and a short trajectory
through the reference's step / corrector loop.  FP64 throughout; the bar
is 1e-12 relative L2 per call and 1e-10 for trajectories.
"""

import numpy as np
import pytest

from conftest import GOLDEN_CASES, load_golden, package_params, rel_l2

pytestmark = pytest.mark.gpu

CALL_TOL = 1e-12
TRAJ_TOL = 1e-10


def make_flow(case, max_iter=10):
    p = package_params(case, max_iter)
    if case["system"] == "plane-couette":
        from dnsjax_b200.flows.plane_couette import PlaneCouetteFlow

        return PlaneCouetteFlow(p)
    from dnsjax_b200.flows.monochromatic import TriplyPeriodicFlow

    return TriplyPeriodicFlow(p, ly=case["ly"])


def dev(a):
    import torch

    return torch.as_tensor(np.ascontiguousarray(a), device="cuda")


def host(t):
    return t.detach().cpu().numpy()


@pytest.fixture(scope="module", params=GOLDEN_CASES)
def setup(request):
    case, g = load_golden(request.param)
    return case, g, make_flow(case)


def test_transforms(setup):
    case, g, flow = setup
    phys = flow.spec_to_phys(dev(g["u0"]))
    assert rel_l2(host(phys), g["phys0"]) < CALL_TOL
    back = flow.phys_to_spec(phys)
    assert rel_l2(host(back), g["u0"]) < CALL_TOL


def test_rhs(setup):
    case, g, flow = setup
    assert rel_l2(host(flow.get_rhs(dev(g["u0"]))), g["rhs0"]) < CALL_TOL
    assert rel_l2(host(flow.get_rhs(dev(g["pred0"]))), g["rhs1"]) < CALL_TOL


def test_predict_correct_norm(setup):
    case, g, flow = setup
    u0, r0, p0, r1 = (dev(g[k]) for k in ("u0", "rhs0", "pred0", "rhs1"))
    assert rel_l2(host(flow.predict(u0, r0)), g["pred0"]) < CALL_TOL
    new, corr = flow.correct(u0, p0, r0, r1)
    assert rel_l2(host(new), g["corr_state0"]) < CALL_TOL
    # The correction is a small difference of O(1) states: its error is
    # bounded relative to the state, not to itself.
    scale = np.linalg.norm(g["corr_state0"])
    assert np.linalg.norm(host(corr) - g["corr0"]) < CALL_TOL * scale
    n0 = float(g["norm0"])
    nscale = float(flow.norm(dev(g["corr_state0"])).item())
    assert abs(float(flow.norm(corr).item()) - n0) <= CALL_TOL * nscale
    import torch

    err = torch.empty(1, dtype=torch.float64, device="cuda")
    fused = flow.correct_fused(u0, p0.clone(), r0, r1, err)
    assert rel_l2(host(fused), g["corr_state0"]) < CALL_TOL
    assert abs(float(err.item()) - n0) <= CALL_TOL * nscale


def test_correct_velocity_and_stats(setup):
    case, g, flow = setup
    u = dev(g["u0"]).clone()
    out, _ = flow.correct_velocity(u)
    assert rel_l2(host(out), g["cv0"]) < CALL_TOL
    if "stats0" in g:
        st = flow.get_stats(dev(g["u0"]))
        np.testing.assert_allclose(list(st.values()), g["stats0"], rtol=1e-12)


@pytest.mark.parametrize("fused", [True, False])
def test_trajectory(setup, fused):
    from dnsjax_b200 import driver

    case, g, flow = setup
    res = driver.run(flow, dev(g["u0"]), case["steps"], fused=fused)
    assert res.corrector_iterations == list(g["iters"])
    assert rel_l2(host(res.state), g["uN"]) < TRAJ_TOL
    np.testing.assert_allclose(res.errors, g["errors"], rtol=1e-6)


@pytest.mark.parametrize("name", [c for c in GOLDEN_CASES if c.startswith("couette")])
def test_couette_imm_unpaired(name, monkeypatch):
    """The IMM kernel without the (kz, -kz) factor sharing gives the same."""
    monkeypatch.setenv("DNSB_IMM_PAIRS", "0")
    case, g = load_golden(name)
    flow = make_flow(case)
    u0, r0, p0, r1 = (dev(g[k]) for k in ("u0", "rhs0", "pred0", "rhs1"))
    assert rel_l2(host(flow.predict(u0, r0)), g["pred0"]) < CALL_TOL
    new, _ = flow.correct(u0, p0, r0, r1)
    assert rel_l2(host(new), g["corr_state0"]) < CALL_TOL
