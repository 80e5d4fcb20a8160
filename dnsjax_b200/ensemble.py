"""Ensembles of independent trajectories advanced in lockstep on one GPU.

Three drivers share the per-trajectory semantics below:

* ``worklist=True`` (periodic members): one CUDA graph per ensemble step
  in which every stage is one launch over all members' blocks
  (``dnsb_ensemble_*``), with a device-controlled corrector loop that runs
  while any member iterates;
* ``graphs=True``: one step graph per member, each on its own stream (the
  fastest measured: members' stages overlap freely, and each member's pass
  buffers stay in L2 between its passes);
* neither: the host-driven lockstep loop.


Each trajectory keeps its own flow context (its own workspace and sizes, so
resolutions may differ) and runs on its own CUDA stream; every time step
follows the reference driver's semantics per trajectory
(src/dnsjax/__main__.py:125-203: predictor + corrector, corrector
iterations until the error is below the tolerance or the cap is reached,
then ``correct_velocity``).  The ensemble enqueues one corrector round for
every still-iterating trajectory before it synchronises once and reads all
their errors, so the kernels of different trajectories overlap on the GPU
and the host waits once per round instead of once per trajectory and
iteration.
"""

from __future__ import annotations

from dataclasses import dataclass, field


@dataclass
class EnsembleStep:
    corrector_iterations: list = field(default_factory=list)
    errors: list = field(default_factory=list)


class Ensemble:
    """autotune=True: the pass variants of every member are picked by timing
    (one tuning per distinct size; see flow.autotune).

    graphs=True: every trajectory's step is one CUDA graph
    launch (predictor, device-controlled corrector loop, correct_velocity;
    see timestep.StepGraph), and the host synchronises once per ensemble step to read
    every trajectory's iterations and error."""

    def __init__(self, flows, states, tol=None, max_iter=None, graphs=False, autotune=False,
                 worklist=False, unroll=None):
        import torch

        if len(flows) != len(states):
            raise ValueError("one state per flow")
        self.flows = list(flows)
        self.states = [s.contiguous() for s in states]
        self.tol = [f.params.step.corrector_tolerance if tol is None else tol
                    for f in self.flows]
        self.max_iter = [f.params.step.max_corrector_iterations if max_iter is None
                         else max_iter for f in self.flows]
        # autotune: pass variants timed once per distinct member size (the
        # first member of each size), shared by the others of that size,
        # before any step graph is captured
        self.tuning = {}
        if autotune:
            for f, st in zip(self.flows, self.states):
                key = (type(f).__name__, f.nx, f.ny, f.nz, bool(getattr(f, "rhs_fp32", False)))
                if key in self.tuning:
                    f.set_variants(self.tuning[key]["variants"])
                else:
                    self.tuning[key] = f.autotune(st)
        self.steppers = [f.make_stepper() for f in self.flows]
        self.streams = [torch.cuda.Stream() for _ in self.flows]
        self.graphs = None
        if graphs and not worklist:
            self.set_unroll(unroll)
        self._ens = None
        if worklist:
            from . import _lib

            if autotune:
                raise ValueError("the work-list ensemble runs the default pass variants")
            L = _lib.lib()
            n = len(self.flows)
            for f in self.flows:
                if not hasattr(f, "make_step_graph") or hasattr(f, "imm"):
                    raise ValueError("the work-list ensemble is built for the periodic flows")
            dbg = self.flows[0].params.debug
            divergence = True if dbg is None else dbg.correct_divergence
            ctxs = (_lib.C.c_void_p * n)(*[f._ctx.value for f in self.flows])
            sts = (_lib.C.c_void_p * n)(*[f._check(x) for f, x in zip(self.flows, self.states)])
            tols = (_lib.C.c_double * n)(*[float(t) for t in self.tol])
            mis = (_lib.C.c_int * n)(*[int(m) for m in self.max_iter])
            h = _lib.C.c_void_p()
            _lib.check(L.dnsb_ensemble_create(ctxs, sts, n, tols, mis, int(divergence),
                                              _lib.C.byref(h)))
            self._ens, self._L = h, L

    def close(self):
        if getattr(self, "_ens", None) is not None and self._ens.value:
            self._L.dnsb_ensemble_destroy(self._ens)
            self._ens = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _worklist_step(self) -> EnsembleStep:
        from . import _lib

        n = len(self.flows)
        _lib.check(self._L.dnsb_ensemble_step(self._ens, _lib.stream_handle()))
        its = (_lib.C.c_int * n)()
        errs = (_lib.C.c_double * n)()
        _lib.check(self._L.dnsb_ensemble_status(self._ens, its, errs, _lib.stream_handle()))
        return EnsembleStep(corrector_iterations=list(its), errors=list(errs))

    def _graph_step(self) -> EnsembleStep:
        import torch

        ready = torch.cuda.current_stream().record_event()
        for g, st in zip(self.graphs, self.streams):
            st.wait_event(ready)
            g.launch(st)
        for st in self.streams:
            torch.cuda.current_stream().wait_stream(st)
        torch.cuda.synchronize()
        res = EnsembleStep()
        for g, st in zip(self.graphs, self.streams):
            it, e = g.status(st)
            res.corrector_iterations.append(it)
            res.errors.append(e)
        return res

    def step_host(self, host_in, host_out) -> EnsembleStep:
        """One ensemble step from pinned host memory to pinned host memory
        (``host_in[i]`` / ``host_out[i]``: member i's state, which may be the
        same buffer): member i's copy-in, step graph and copy-out run in that
        order on member i's stream, so the copies of some members overlap the
        steps of others.  Needs the step-graph form (``graphs=True``)."""
        import torch

        if self.graphs is None:
            raise ValueError("step_host runs the step-graph form (graphs=True)")
        ready = torch.cuda.current_stream().record_event()
        for g, st, x, hi, ho in zip(self.graphs, self.streams, self.states, host_in, host_out):
            st.wait_event(ready)
            with torch.cuda.stream(st):
                x.copy_(hi, non_blocking=True)  # the graph is bound to x
            g.launch(st)
            with torch.cuda.stream(st):
                ho.copy_(x, non_blocking=True)
        for st in self.streams:
            torch.cuda.current_stream().wait_stream(st)
        torch.cuda.synchronize()
        res = EnsembleStep()
        for g, st in zip(self.graphs, self.streams):
            it, e = g.status(st)
            res.corrector_iterations.append(it)
            res.errors.append(e)
        return res

    def set_unroll(self, unroll) -> None:
        """(Re)captures every member's step graph with ``unroll`` corrector
        iterations held as straight-line kernels (None: the flows' own
        setting; see make_step_graph)."""
        for g in self.graphs or []:
            g.close()
        self.graphs = [f.make_step_graph(s, tol=t, max_iter=m, unroll=unroll)
                       for f, s, t, m in zip(self.flows, self.states, self.tol, self.max_iter)]

    def step(self) -> EnsembleStep:
        import torch

        if self._ens is not None:
            return self._worklist_step()
        if self.graphs is not None:
            return self._graph_step()

        n = len(self.flows)
        prev = list(self.states)
        cur, rhs, err = [None] * n, [None] * n, [None] * n
        # record on the current stream so every trajectory stream sees the
        # states produced before this call
        ready = torch.cuda.current_stream().record_event()
        for i in range(n):
            with torch.cuda.stream(self.streams[i]):
                self.streams[i].wait_event(ready)
                cur[i], rhs[i], err[i] = self.steppers[i][0](prev[i])
        torch.cuda.synchronize()
        e = [float(x.item()) for x in err]
        iters = [0] * n
        active = [i for i in range(n) if e[i] > self.tol[i] and iters[i] < self.max_iter[i]]
        while active:
            for i in active:
                with torch.cuda.stream(self.streams[i]):
                    cur[i], rhs[i], err[i] = self.steppers[i][1](prev[i], cur[i], rhs[i])
                iters[i] += 1
            torch.cuda.synchronize()
            for i in active:
                e[i] = float(err[i].item())
            active = [i for i in active
                      if e[i] > self.tol[i] and iters[i] < self.max_iter[i]]
        for i in range(n):
            with torch.cuda.stream(self.streams[i]):
                cur[i], _ = self.flows[i].correct_velocity(cur[i])
        done = [s.record_event() for s in self.streams]
        for ev in done:
            torch.cuda.current_stream().wait_event(ev)
        self.states = cur
        return EnsembleStep(corrector_iterations=iters, errors=e)
