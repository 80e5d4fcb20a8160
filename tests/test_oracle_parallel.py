"""The oracle's thread-parallel slices give bitwise the serial results.

oracle/parallel.py splits FFT lines, y-stencils and banded solves over
threads. Each slice computes its lines or modes exactly as the whole call
does. Here one RHS and one corrector of a plane-Couette field (32x33x32,
p = 4) and of a Kolmogorov field (24^3) are computed with 1 and with 4
threads, and must agree bit for bit.
"""

from math import pi

import numpy as np

from oracle import parallel
from oracle.config import Config


def _rhs_and_correct(S, u0):
    r0 = S.get_rhs(u0)
    new, corr = S.correct(u0, u0, r0, r0)
    return r0, new, corr, S.norm(corr)


def _both(S, u0):
    try:
        parallel.set_threads(1)
        serial = _rhs_and_correct(S, u0)
        parallel.set_threads(4)
        threaded = _rhs_and_correct(S, u0)
    finally:
        parallel.set_threads(1)
    return serial, threaded


def test_couette_threads_bitwise():
    from dnsjax_b200 import initial
    from oracle.couette import CouetteSetup

    cfg = Config(system="plane-couette", nx=32, ny=33, nz=32, lx=2 * pi, lz=pi, re=400.0,
                 dt=0.02, corrector_tolerance=1e-10, fd_order=4)
    S = CouetteSetup(cfg)
    u0 = initial.couette_field(32, 33, 32, 2 * pi, pi, 4, 3, 8.0, 1e-3)
    serial, threaded = _both(S, u0)
    for a, b in zip(serial, threaded):
        assert np.array_equal(a, b)


def test_periodic_threads_bitwise():
    from dnsjax_b200 import initial
    from oracle.periodic import PeriodicSetup

    cfg = Config(system="kolmogorov", nx=24, ny=24, nz=24, lx=2 * pi, ly=2 * pi, lz=2 * pi,
                 re=40.0, dt=0.01, corrector_tolerance=1e-10)
    S = PeriodicSetup(cfg)
    u0 = initial.periodic_field(24, 24, 24, 2 * pi, 2 * pi, 2 * pi, 5,
                                initial.kolmogorov_spectrum_k53, 0.1)
    serial, threaded = _both(S, u0)
    for a, b in zip(serial, threaded):
        assert np.array_equal(a, b)


def test_split_falls_back_to_the_serial_call():
    parallel.set_threads(4)
    try:
        x = np.arange(6.0).reshape(3, 2)
        # 3 rows make one slice of at least 2 rows: the serial call
        assert np.array_equal(parallel.split(lambda a: a * 2, (x,), 0), x * 2)
        # 5 rows make two slices (not four)
        y = np.arange(10.0).reshape(5, 2)
        sizes = []
        parallel.split(lambda a: sizes.append(a.shape[0]) or a, (y,), 0)
        assert sorted(sizes) == [2, 3]
    finally:
        parallel.set_threads(1)
    assert parallel.threads() == 1
