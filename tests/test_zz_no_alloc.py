"""dnsb_couette_norm_noalloc: the allocation-free Couette norm.

Callers that cannot allocate device memory -- such as an XLA FFI handler
working in memory its framework owns -- cannot create a dnsb_couette context either; this entry point gives them the same
norm from the field alone, keeping its partial sums in a fixed-size array
inside the library.  It must agree with the context-based dnsb_couette_norm
call after call (the array keeps the previous call's contents, which must
never leak into the next result).  This file is collected last.
"""

import ctypes
from math import pi

import pytest


def _flow(nx, ny, nz, p):
    from dnsjax_b200.flows.plane_couette import PlaneCouetteFlow
    from dnsjax_b200.parameters import Parameters

    params = Parameters(phys=dict(system="plane-couette", re=400.0),
                        geo=dict(lx=2 * pi, lz=pi),
                        res=dict(nx=nx, ny=ny, nz=nz, fd_order=p),
                        step=dict(dt=0.02))
    return PlaneCouetteFlow(params)


@pytest.mark.gpu
def test_noalloc_norm_matches_context_norm_twice():
    import torch

    from dnsjax_b200 import _lib, initial

    L = _lib.lib()
    out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    # first a larger field, then a smaller one: the second result must not
    # see the first call's partial sums
    for (nx, ny, nz, p, seed, energy) in ((16, 33, 12, 4, 3, 1e-2),
                                          (8, 17, 8, 4, 4, 0.5)):
        flow = _flow(nx, ny, nz, p)
        v = torch.as_tensor(initial.couette_field(nx, ny, nz, 2 * pi, pi, p,
                                                  seed, 8.0, energy),
                            device="cuda")
        ref = float(flow.norm(v).item())
        _lib.check(L.dnsb_couette_norm_noalloc(
            _lib.ptr(v), nx, ny, nz, 2.0, _lib.ptr(out), _lib.stream_handle()))
        got = float(out.item())
        assert abs(got - ref) <= 1e-12 * ref, (got, ref)


@pytest.mark.gpu
def test_noalloc_norm_at_the_mode_limit_and_tall_grid():
    """Near the 32768-mode limit with a mode count that leaves the last
    block of warps partly filled (129 x 253 = 32637 modes, not a multiple of
    the four modes per block), and the 129-point grid of the 128x129x128
    workload (odd and even Simpson panels at both walls): against the
    oracle's Simpson norm at 1e-12, and the 128x129x128 field also against
    the context norm, each twice in a row."""
    import numpy as np
    import torch

    from dnsjax_b200 import _lib, initial
    from oracle.couette import cgl_grid, simpson_weights_apply

    L = _lib.lib()
    out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")

    def noalloc(v, nx, ny, nz):
        _lib.check(L.dnsb_couette_norm_noalloc(
            _lib.ptr(v), nx, ny, nz, 2.0, _lib.ptr(out), _lib.stream_handle()))
        return float(out.item())

    def oracle_norm(vh, nx, ny):
        km = np.where(np.arange(nx // 2) == 0, 1.0, 2.0).reshape(1, 1, -1, 1)
        prof = np.sum((np.conj(vh) * km * vh).real, axis=(0, 1, 2))
        return float(np.sqrt(simpson_weights_apply(prof, cgl_grid(ny)) / 2.0))

    nx, ny, nz = 258, 129, 254
    assert (nz - 1) * (nx // 2) == 32637 and 32637 % 4 != 0
    rng = np.random.default_rng(5)
    shape = (3, nz - 1, nx // 2, ny)
    vh = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    v = torch.as_tensor(vh, device="cuda")
    ref = oracle_norm(vh, nx, ny)
    for _ in range(2):
        got = noalloc(v, nx, ny, nz)
        assert abs(got - ref) <= 1e-12 * ref, (got, ref)
    del v

    nx, ny, nz = 128, 129, 128
    flow = _flow(nx, ny, nz, 6)
    vh = initial.couette_field(nx, ny, nz, 2 * pi, pi, 6, 4, 32.0, 5e-2)
    v = torch.as_tensor(vh, device="cuda")
    ref = float(flow.norm(v).item())
    assert abs(ref - oracle_norm(vh, nx, ny)) <= 1e-12 * ref
    for _ in range(2):
        got = noalloc(v, nx, ny, nz)
        assert abs(got - ref) <= 1e-12 * ref, (got, ref)


def test_noalloc_rejects_fields_beyond_its_scratch():
    """(nz-1)*(nx/2) above 32768 modes is refused before any GPU work."""
    from dnsjax_b200 import _lib, build

    build.build()
    h = _lib.load()
    rc = h.dnsb_couette_norm_noalloc(ctypes.c_void_p(16), 512, 129, 512, 2.0,
                                     ctypes.c_void_p(16), None)
    assert rc == 1  # DNSB_ERR_ARG
    assert b"32768" in h.dnsb_last_error()
