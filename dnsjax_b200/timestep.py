"""Predictor-corrector stepper factory (the reference's make_stepper contract).

``make_stepper(get_rhs_fn, predict_fn, correct_fn, norm_fn)`` returns
``predict_and_correct(state) -> (prediction, rhs_next, error)`` and
``iterate_correction(state_prev, prediction, rhs_prev) -> (prediction,
rhs_next, error)`` exactly as src/dnsjax/timestep.py:23-122 composes them
(Euler predictor, then Crank-Nicolson corrector iterations; the caller
passes the previous iterate's RHS as ``rhs_prev``).  Extra positional
arguments are forwarded to the callables, as the reference forwards
``(fourier, flow)``.

``make_fused_stepper(flow)`` is the same contract over a flow object whose
``correct_fused`` applies the corrector and reduces the correction norm in
one kernel (the correction is never stored) and updates the donated
prediction in place -- what ``donate_argnums=1`` allows in the reference.
The error is a 1-element float64 device tensor; comparing it with the
tolerance on the host is the only synchronisation per corrector iteration,
as in the reference driver (src/dnsjax/__main__.py:167-170).
"""

from __future__ import annotations

from collections.abc import Callable


def make_stepper(get_rhs_fn: Callable, predict_fn: Callable,
                 correct_fn: Callable, norm_fn: Callable):
    def predict_and_correct(state, *args):
        rhs_prev = get_rhs_fn(state, *args)
        prediction = predict_fn(state, rhs_prev, *args)
        rhs_next = get_rhs_fn(prediction, *args)
        prediction, correction = correct_fn(state, prediction, rhs_prev,
                                            rhs_next, *args)
        return prediction, rhs_next, norm_fn(correction, *args)

    def iterate_correction(state_prev, prediction, rhs_prev, *args):
        rhs_next = get_rhs_fn(prediction, *args)
        prediction, correction = correct_fn(state_prev, prediction, rhs_prev,
                                            rhs_next, *args)
        return prediction, rhs_next, norm_fn(correction, *args)

    return predict_and_correct, iterate_correction


def make_fused_stepper(flow):
    import torch

    def _err():
        return torch.empty(1, dtype=torch.float64, device="cuda")

    def predict_and_correct(state):
        rhs_prev = flow.get_rhs(state)
        prediction = flow.predict(state, rhs_prev)
        rhs_next = flow.get_rhs(prediction)
        err = _err()
        prediction = flow.correct_fused(state, prediction, rhs_prev, rhs_next,
                                        err, out=prediction)
        return prediction, rhs_next, err

    def iterate_correction(state_prev, prediction, rhs_prev):
        rhs_next = flow.get_rhs(prediction)
        err = _err()
        prediction = flow.correct_fused(state_prev, prediction, rhs_prev,
                                        rhs_next, err, out=prediction)
        return prediction, rhs_next, err

    return predict_and_correct, iterate_correction


class StepGraph:
    """One full time step (predictor, device-controlled corrector loop,
    correct_velocity) captured as a CUDA graph on a flow's context; every
    launch advances the bound state in place without host synchronisation.
    status() returns the corrector iterations and error of the last step.
    ``create(handle_ref)`` is the flow's dnsb_*_step_graph_create call."""

    def __init__(self, lib, state, create):
        from . import _lib

        self._L, self.state = lib, state
        h = _lib.C.c_void_p()
        _lib.check(create(_lib.C.byref(h)))
        self._h = h

    def launch(self, stream=None):
        from . import _lib

        _lib.check(self._L.dnsb_step_graph_launch(self._h, _lib.stream_handle(stream)))

    def status(self, stream=None):
        from . import _lib

        it, err = _lib.C.c_int(), _lib.C.c_double()
        _lib.check(self._L.dnsb_step_graph_status(
            self._h, _lib.C.byref(it), _lib.C.byref(err), _lib.stream_handle(stream)))
        return it.value, err.value

    def close(self):
        if getattr(self, "_h", None):
            self._L.dnsb_step_graph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
