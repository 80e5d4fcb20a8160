"""The oracle against golden vectors from the reference's own source.

The fixtures in tests/golden were produced by running the reference solver
(src/dnsjax) through a NumPy-backed stand-in for jax
(tests/golden/make_golden.py).  The oracle restates the same arithmetic, so
agreement is expected to rounding level (observed: bit-identical).
"""

import numpy as np
import pytest

from conftest import (COUETTE_CASES, GOLDEN_CASES, load_golden, oracle_config,
                      rel_l2)

TOL = 1e-12


def _setup(case):
    from oracle.couette import CouetteSetup
    from oracle.periodic import PeriodicSetup

    cfg = oracle_config(case)
    return cfg, (CouetteSetup(cfg) if cfg.system == "plane-couette"
                 else PeriodicSetup(cfg))


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_single_calls(name):
    from oracle import fft as F

    case, g = load_golden(name)
    cfg, S = _setup(case)
    u0 = g["u0"]
    phys = (F.spec_to_phys_2d(u0, cfg) if cfg.system == "plane-couette"
            else F.spec_to_phys(u0, cfg))
    assert rel_l2(phys, g["phys0"]) < TOL
    r0 = S.get_rhs(u0)
    assert rel_l2(r0, g["rhs0"]) < TOL
    p0 = S.predict(u0, r0)
    assert rel_l2(p0, g["pred0"]) < TOL
    r1 = S.get_rhs(p0)
    assert rel_l2(r1, g["rhs1"]) < TOL
    cs, cc = S.correct(u0, p0, r0, r1)
    assert rel_l2(cs, g["corr_state0"]) < TOL
    assert rel_l2(cc, g["corr0"]) < TOL
    assert abs(S.norm(cc) - float(g["norm0"])) <= TOL * float(g["norm0"])
    cv = S.correct_velocity(u0)
    assert rel_l2(cv, g["cv0"]) < TOL
    if "stats0" in g:
        st = S.stats(u0)
        np.testing.assert_allclose(list(st.values()), g["stats0"], rtol=1e-12)


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_trajectory(name):
    from oracle.stepper import run

    case, g = load_golden(name)
    cfg, S = _setup(case)
    res = run(S, g["u0"], case["steps"])
    assert res.corrector_iterations == list(g["iters"])
    assert rel_l2(res.state, g["uN"]) < TOL
    np.testing.assert_allclose(res.errors, g["errors"], rtol=1e-9)


@pytest.mark.parametrize("name", COUETTE_CASES)
def test_imm_precompute(name):
    """The oracle's precompute_imm reproduces the reference's arrays."""
    case, g = load_golden(name)
    _, S = _setup(case)
    for k in ("Lk_ab", "Hk_ab", "p1", "p2", "v1", "v2", "q1", "q2", "M_inv",
              "D1", "D2"):
        np.testing.assert_allclose(S.imm[k], g[k], rtol=1e-12, atol=1e-12 *
                                   max(1.0, float(np.abs(g[k]).max())), err_msg=k)
    np.testing.assert_array_equal(S.imm["Lk_piv"], g["Lk_piv"])
    np.testing.assert_array_equal(S.imm["Hk_piv"], g["Hk_piv"])


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_snapshot_read_by_the_reference(name):
    """The snapshot file the fixture generator wrote from u0 and read back
    with the reference's own init_state: the oracle's forward transform of
    the file's array (minus the base flow for the periodic flows) is the
    state the reference read, and that state is u0 to rounding."""
    from oracle import fft as F

    case, g = load_golden(name)
    cfg, S = _setup(case)
    snap = g["snapshot_phys"]
    if cfg.system == "plane-couette":
        spec = F.phys_to_spec_2d(snap, cfg)
    else:
        spec = F.phys_to_spec(snap - S.base_flow, cfg)
    assert rel_l2(spec, g["snapshot_loaded"]) < TOL
    assert rel_l2(g["snapshot_loaded"], g["u0"]) < 1e-12
