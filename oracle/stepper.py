"""Predictor-corrector stepper and driver loop (oracle; test infra only).

``make_stepper`` restates ``src/dnsjax/timestep.py:23-122``; ``run``
restates the step/corrector loop of ``src/dnsjax/__main__.py:125-203``
(corrector bound, termination on a non-converged step, and the
``rhs_prev`` hand-over between corrector iterations).
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


def make_stepper(get_rhs, predict, correct, norm):
    """timestep.py:23-122."""

    def predict_and_correct(state):
        rhs_prev = get_rhs(state)
        pred = predict(state, rhs_prev)
        rhs_next = get_rhs(pred)
        pred, corr = correct(state, pred, rhs_prev, rhs_next)
        return pred, rhs_next, norm(corr)

    def iterate_correction(state_prev, pred, rhs_prev):
        rhs_next = get_rhs(pred)
        pred, corr = correct(state_prev, pred, rhs_prev, rhs_next)
        return pred, rhs_next, norm(corr)

    return predict_and_correct, iterate_correction


@dataclass
class RunResult:
    state: np.ndarray
    steps: int
    corrector_iterations: list = field(default_factory=list)
    errors: list = field(default_factory=list)
    converged: bool = True


def run(setup, state, steps: int) -> RunResult:
    """__main__.py:125-203 for a fixed number of steps."""
    cfg = setup.cfg
    pac, itc = make_stepper(setup.get_rhs, setup.predict, setup.correct,
                            setup.norm)
    res = RunResult(state=state, steps=0)
    last_error = 0.0
    for _ in range(steps):
        if not last_error < cfg.corrector_tolerance:
            res.converged = False
            break
        state_prev = state
        state, rhs, err = pac(state_prev)
        c = 0
        while err > cfg.corrector_tolerance and c < cfg.max_corrector_iterations:
            state, rhs, err = itc(state_prev, state, rhs)
            c += 1
        state = setup.correct_velocity(state, cfg.correct_divergence)
        last_error = err
        res.steps += 1
        res.corrector_iterations.append(c)
        res.errors.append(err)
    res.state = state
    if not last_error < cfg.corrector_tolerance and res.steps:
        res.converged = False
    return res
