"""Host logic of the stepper factory and the driver loop (no GPU).

A fake flow with scalar "states" checks the call sequence of
make_stepper (timestep.py:23-122 of the reference) and the loop rules of
__main__.py:125-203: corrector bound, rhs_prev hand-over, stop on failure.
"""

import numpy as np

from dnsjax_b200 import driver
from dnsjax_b200.parameters import Parameters
from dnsjax_b200.timestep import make_stepper


class _Err:
    def __init__(self, v):
        self.v = v

    def item(self):
        return self.v


class FakeFlow:
    """x' = contraction towards 1 with rate r; error = |correction|."""

    def __init__(self, rate, tol=1e-10, max_iter=10):
        self.params = Parameters(step=dict(corrector_tolerance=tol,
                                           max_corrector_iterations=max_iter))
        self.rate = rate
        self.calls = []

    def get_rhs(self, s):
        self.calls.append(("rhs", s))
        return s

    def predict(self, s, r):
        return s + 2.0

    def correct(self, sp, pred, rp, rn):
        self.calls.append(("correct", rp, rn))
        new = 1.0 + self.rate * (pred - 1.0)
        return new, new - pred

    def norm(self, c):
        return _Err(abs(c))

    def correct_velocity(self, s):
        return s, None

    def make_stepper(self, fused=True):
        return make_stepper(self.get_rhs, self.predict, self.correct, self.norm)


def test_rhs_prev_is_previous_iterate():
    f = FakeFlow(0.5)
    pac, itc = f.make_stepper()
    s1, r1, e1 = pac(0.0)
    s2, r2, e2 = itc(0.0, s1, r1)
    corr = [c for c in f.calls if c[0] == "correct"]
    # second corrector receives the first corrector's rhs_next as rhs_prev
    assert corr[1][1] == corr[0][2]


def test_loop_bounds_and_stop():
    f = FakeFlow(0.5, tol=1e-3, max_iter=3)
    res = driver.run(f, 0.0, steps=5, fused=False)
    # 1 - 0.5^k below 1e-3 needs k = 10 > 1 + 3: the first step fails
    assert res.steps == 1 and res.corrector_iterations == [3]
    assert not res.converged
    f = FakeFlow(0.01, tol=1e-3, max_iter=3)
    res = driver.run(f, 0.0, steps=4, fused=False)
    assert res.steps == 4 and res.converged
    assert all(c <= 3 for c in res.corrector_iterations)
    res = driver.run(FakeFlow(0.5, 1e-3, 3), 0.0, steps=3, fused=False,
                     stop_on_failure=False)
    assert res.steps == 3 and not res.converged


def test_oracle_stepper_same_sequence():
    from oracle.stepper import make_stepper as omake

    f1, f2 = FakeFlow(0.3), FakeFlow(0.3)
    a = make_stepper(f1.get_rhs, f1.predict, f1.correct, f1.norm)
    b = omake(f2.get_rhs, f2.predict, f2.correct, lambda c: abs(c))
    x1, r1, _ = a[0](0.0)
    x2, r2, _ = b[0](0.0)
    assert np.isclose(x1, x2) and f1.calls == f2.calls


def test_non_finite_error_ends_the_run():
    """A NaN correction norm: no corrector iteration (NaN > tol is false), and
    the loop stops before the next step (not NaN < tol), as
    __main__.py:125-129 does."""
    f = FakeFlow(0.5, tol=1e-3, max_iter=3)
    res = driver.run(f, float("nan"), steps=5, fused=False)
    assert res.steps == 1 and res.corrector_iterations == [0]
    assert not res.converged and np.isnan(res.errors[0])
