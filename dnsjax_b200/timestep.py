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

    def run_host(self, host_in, host_out, chunks: int = 4):
        """One step from pinned host memory to pinned host memory: the state
        copied in, the step graph launched, the new state copied out, all
        ordered on the current stream's timeline without host waits.

        The copies move in ``chunks`` pieces on two copy streams.  When
        ``host_in`` is the ``host_out`` of the previous call (a trajectory
        that round-trips through the host every step), piece i of this
        copy-in starts as soon as piece i of the previous copy-out has
        landed, so the two directions of the link overlap instead of
        running one after the other.  ``host_out`` is complete once
        ``wait_host()`` has ordered the current stream after the copy-out
        and that stream has been synchronized."""
        import torch

        main = torch.cuda.current_stream()
        if getattr(self, "_copy_streams", None) is None:
            self._copy_streams = (torch.cuda.Stream(), torch.cuda.Stream())
            self._out_events, self._out_ptr = [], None
        s_in, s_out = self._copy_streams
        d = self.state.view(-1)
        hi, ho = host_in.view(-1), host_out.view(-1)
        n = d.numel()
        bounds = [(n * i) // chunks for i in range(chunks + 1)]
        # host_in still being written by the previous copy-out: piece by
        # piece when the pieces match, else after all of it
        chained = self._out_ptr == host_in.data_ptr()
        per_piece = chained and len(self._out_events) == chunks
        if chained and not per_piece:
            s_in.wait_event(self._out_events[-1])
        s_in.wait_stream(main)  # the previous step's graph no longer reads the state
        for i in range(chunks):
            a, b = bounds[i], bounds[i + 1]
            if per_piece:
                s_in.wait_event(self._out_events[i])
            with torch.cuda.stream(s_in):
                d[a:b].copy_(hi[a:b], non_blocking=True)
        main.wait_stream(s_in)
        self.launch(main)
        s_out.wait_stream(main)
        events = []
        for i in range(chunks):
            a, b = bounds[i], bounds[i + 1]
            with torch.cuda.stream(s_out):
                ho[a:b].copy_(d[a:b], non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(s_out)
            events.append(ev)
        self._out_events, self._out_ptr = events, host_out.data_ptr()

    def wait_host(self) -> None:
        """Orders the current stream after the last run_host copy-out."""
        import torch

        if getattr(self, "_out_events", None):
            torch.cuda.current_stream().wait_event(self._out_events[-1])

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
