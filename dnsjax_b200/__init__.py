"""dnsjax_b200: B200-native (sm_100a) time-step hot path for dnsjax.

The package mirrors the reference solver's time-step interface
(gokhanyalniz/dnsjax): ``timestep.make_stepper`` and the per-flow
``predict_and_correct`` / ``iterate_correction`` / ``correct_velocity`` /
``get_stats`` / ``init_state`` functions, selected by
``params.solver.backend = "cuda"``.  All time-step arithmetic runs in the
hand-written CUDA kernels of ``libdnsb.so`` (``dnsjax_b200/csrc``), reached
through the C ABI declared in ``include/dnsb.h``.  There is no CPU path: if
the library or a GPU is missing, the flow objects raise.
"""

__all__ = ["parameters", "timestep"]
