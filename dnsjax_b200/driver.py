"""Time-step loop with the reference driver's semantics.

Restates the step / corrector loop of src/dnsjax/__main__.py:125-203 over a
flow object: each step is ``predict_and_correct``, then
``iterate_correction`` while ``error > corrector_tolerance`` and fewer than
``max_corrector_iterations`` extra iterations ran (passing the previous
iterate's RHS as ``rhs_prev``), then ``correct_velocity``.  As in the
reference, a step that ends above the tolerance ends the run
(``stop_on_failure``); benchmarks may keep stepping to measure throughput.
"""

from __future__ import annotations

from dataclasses import dataclass, field


@dataclass
class RunResult:
    state: object
    steps: int = 0
    corrector_iterations: list = field(default_factory=list)
    errors: list = field(default_factory=list)
    converged: bool = True


def step(flow, steppers, state, tol: float, max_iter: int):
    """One time step; returns (state, corrector iterations, error)."""
    pac, itc = steppers
    state_prev = state
    state, rhs, err = pac(state_prev)
    c = 0
    e = float(err.item())
    while e > tol and c < max_iter:
        state, rhs, err = itc(state_prev, state, rhs)
        c += 1
        e = float(err.item())
    state, _ = flow.correct_velocity(state)
    return state, c, e


def run(flow, state, steps: int, tol: float | None = None,
        max_iter: int | None = None, stop_on_failure: bool = True,
        fused: bool = True) -> RunResult:
    p = flow.params
    tol = p.step.corrector_tolerance if tol is None else tol
    max_iter = p.step.max_corrector_iterations if max_iter is None else max_iter
    steppers = flow.make_stepper(fused=fused)
    res = RunResult(state=state)
    last_error = 0.0
    for _ in range(steps):
        if stop_on_failure and not last_error < tol:
            break
        state, c, e = step(flow, steppers, state, tol, max_iter)
        last_error = e
        res.steps += 1
        res.corrector_iterations.append(c)
        res.errors.append(e)
        if not e < tol:
            res.converged = False
    res.state = state
    return res
