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


def test_noalloc_rejects_fields_beyond_its_scratch():
    """(nz-1)*(nx/2) above 32768 modes is refused before any GPU work."""
    from dnsjax_b200 import _lib, build

    build.build()
    h = _lib.load()
    rc = h.dnsb_couette_norm_noalloc(ctypes.c_void_p(16), 512, 129, 512, 2.0,
                                     ctypes.c_void_p(16), None)
    assert rc == 1  # DNSB_ERR_ARG
    assert b"32768" in h.dnsb_last_error()
