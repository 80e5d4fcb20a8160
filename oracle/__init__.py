"""CPU oracle for the dnsjax time-step hot path (TEST INFRASTRUCTURE ONLY).

This package is a NumPy/SciPy FP64 restatement of the reference solver's
time-step path (gokhanyalniz/dnsjax, ``src/dnsjax``).  It exists only to
check the CUDA implementation in ``dnsjax_b200``: the tests, the smoke test
and the ``cpu_baseline`` leg of ``bench.py`` may import it, nothing in the
product may.  Every function cites the reference ``file:line`` it follows.

Pinning:

* the banded LU / dgbtrs restatement and the two matrix-free matvecs are
  pinned by the reference's own known-answer tests
  (``tests/test_banded_solver.py``), restated in ``tests/test_oracle_kats.py``;
* the whole step (FFTs, nonlinear term, projection, IMM, predictor,
  corrector, norms, divergence correction, stats) is pinned against golden
  vectors produced by running the reference's own source through a
  NumPy-backed stand-in for the ``jax`` API (``tests/golden/make_golden.py``).
"""
