"""ctypes binding of libdnsb.so (declared in include/dnsb.h).

The shared library is built in-tree (``python -m dnsjax_b200.build``) and
loaded from this package directory.  There is no fallback: if the library is
missing or CUDA is unavailable, :func:`lib` raises.
"""

from __future__ import annotations

import ctypes as C
from pathlib import Path

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "libdnsb.so"

_lib = None

c_int, c_ll, c_double, c_void_p, c_size_t = (
    C.c_int, C.c_longlong, C.c_double, C.c_void_p, C.c_size_t)
P_double = C.POINTER(C.c_double)
P_int = C.POINTER(C.c_int)


class PeriodicDesc(C.Structure):
    _fields_ = [
        ("nx", c_int), ("ny", c_int), ("nz", c_int),
        ("nx_p", c_int), ("ny_p", c_int), ("nz_p", c_int),
        ("dt", c_double), ("implicitness", c_double),
        ("kx", P_double), ("ky", P_double), ("kz", P_double),
        ("base_flow", P_double), ("curl_base_flow", P_double),
        ("nonlin_base_flow", P_double),
        ("ldt_1", P_double), ("ildt_2", P_double),
    ]


class CouetteDesc(C.Structure):
    _fields_ = [
        ("nx", c_int), ("ny", c_int), ("nz", c_int),
        ("nx_p", c_int), ("nz_p", c_int), ("fd_order", c_int),
        ("dt", c_double), ("implicitness", c_double), ("nu", c_double),
        ("ly", c_double),
        ("kx", P_double), ("kz", P_double), ("ys", P_double),
        ("d1_j0", P_int), ("d1_w", P_double),
        ("d2_j0", P_int), ("d2_w", P_double),
        ("base_flow", P_double), ("curl_base_flow", P_double),
        ("nonlin_base_flow", P_double),
    ]


class ImmOps(C.Structure):
    _fields_ = [
        ("Lk_ab", c_void_p), ("Lk_piv", c_void_p),
        ("Hk_ab", c_void_p), ("Hk_piv", c_void_p),
        ("v1", c_void_p), ("v2", c_void_p),
        ("q1", c_void_p), ("q2", c_void_p),
        ("M_inv", c_void_p),
    ]


# name -> (restype, argtypes); every entry point declared in include/dnsb.h
SIGNATURES = {
    "dnsb_version": (c_int, []),
    "dnsb_last_error": (C.c_char_p, []),
    "dnsb_launch_count": (c_ll, []),
    "dnsb_periodic_create": (c_int, [C.POINTER(PeriodicDesc), C.POINTER(c_void_p)]),
    "dnsb_periodic_destroy": (c_int, [c_void_p]),
    "dnsb_periodic_workspace_bytes": (c_size_t, [c_void_p]),
    "dnsb_periodic_rhs": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "dnsb_periodic_predict": (c_int, [c_void_p] * 5),
    "dnsb_periodic_correct": (c_int, [c_void_p] * 8),
    "dnsb_periodic_norm": (c_int, [c_void_p] * 4),
    "dnsb_periodic_correct_velocity": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_void_p]),
    "dnsb_periodic_energy_sums": (c_int, [c_void_p] * 4),
    "dnsb_periodic_step_graph_create": (c_int, [c_void_p, c_void_p, c_double, c_int, c_int,
                                                C.POINTER(c_void_p)]),
    "dnsb_couette_step_graph_create": (c_int, [c_void_p, c_void_p, c_double, c_int,
                                               C.POINTER(c_void_p)]),
    "dnsb_step_graph_launch": (c_int, [c_void_p, c_void_p]),
    "dnsb_step_graph_status": (c_int, [c_void_p, P_int, P_double, c_void_p]),
    "dnsb_step_graph_destroy": (c_int, [c_void_p]),
    "dnsb_couette_set_graph_unroll": (c_int, [c_void_p, c_int]),
    "dnsb_periodic_set_graph_unroll": (c_int, [c_void_p, c_int]),
    "dnsb_couette_mixed_graph_create": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p,
                                                c_double, c_int, c_int, c_double, c_double,
                                                c_int, C.POINTER(c_void_p)]),
    "dnsb_mixed_graph_predict": (c_int, [c_void_p, c_void_p]),
    "dnsb_mixed_graph_correct": (c_int, [c_void_p, c_void_p]),
    "dnsb_mixed_graph_status": (c_int, [c_void_p, P_int, P_double, P_double, P_int, P_int,
                                        c_void_p]),
    "dnsb_mixed_graph_destroy": (c_int, [c_void_p]),
    "dnsb_periodic_spec_to_phys": (c_int, [c_void_p] * 4),
    "dnsb_periodic_phys_to_spec": (c_int, [c_void_p] * 4),
    "dnsb_couette_create": (c_int, [C.POINTER(CouetteDesc), C.POINTER(c_void_p)]),
    "dnsb_couette_destroy": (c_int, [c_void_p]),
    "dnsb_couette_workspace_bytes": (c_size_t, [c_void_p]),
    "dnsb_couette_bind_imm": (c_int, [c_void_p, C.POINTER(ImmOps)]),
    "dnsb_couette_rhs": (c_int, [c_void_p] * 4),
    "dnsb_couette_imm": (c_int, [c_void_p] * 9),
    "dnsb_couette_norm": (c_int, [c_void_p] * 4),
    "dnsb_couette_norm2": (c_int, [c_void_p] * 4),
    "dnsb_couette_spec_to_phys": (c_int, [c_void_p] * 4),
    "dnsb_couette_phys_to_spec": (c_int, [c_void_p] * 4),
    "dnsb_couette_check": (c_int, [c_void_p, c_void_p]),
    "dnsb_ensemble_create": (c_int, [c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_int,
                                     c_void_p]),
    "dnsb_ensemble_step": (c_int, [c_void_p, c_void_p]),
    "dnsb_ensemble_status": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "dnsb_ensemble_destroy": (c_int, [c_void_p]),
    "dnsb_couette_clear_status": (c_int, [c_void_p, c_void_p]),
    "dnsb_couette_set_wait_limit": (c_int, [c_void_p, c_int]),
    "dnsb_periodic_set_rhs_precision": (c_int, [c_void_p, c_int]),
    "dnsb_couette_set_rhs_precision": (c_int, [c_void_p, c_int]),
    "dnsb_periodic_autotune": (c_int, [c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_void_p]),
    "dnsb_couette_autotune": (c_int, [c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_void_p]),
    "dnsb_periodic_set_variants": (c_int, [c_void_p, c_void_p]),
    "dnsb_couette_set_variants": (c_int, [c_void_p, c_void_p]),
    "dnsb_mlp_gemm": (c_int, [c_int, c_int, c_int, c_int, c_int, c_void_p, c_int, c_void_p,
                              c_int, c_void_p, c_int, c_void_p, c_int, c_void_p, c_void_p, c_int,
                              c_void_p, C.c_longlong, c_void_p, c_void_p]),
    "dnsb_mlp_transpose": (c_int, [c_void_p, c_int, c_int, c_int, c_void_p, c_int, c_void_p]),
    "dnsb_learned_features": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_double,
                                      c_double, c_double, c_void_p, c_int, c_void_p, c_int,
                                      c_void_p, c_void_p]),
    "dnsb_learned_guess": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_void_p,
                                   c_void_p]),
    "dnsb_mlp_loss_grad": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_void_p, c_void_p,
                                   c_void_p, c_void_p, c_void_p]),
    "dnsb_mlp_colsum": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_void_p, c_void_p,
                                C.c_longlong, c_void_p]),
    "dnsb_mlp_adam": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, C.c_longlong,
                              C.c_float, C.c_float, C.c_float, C.c_float, c_int, c_void_p]),
    "dnsb_imm_precompute": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_int, c_int,
                                    c_int, c_double, c_double, c_double] + [c_void_p] * 13),
    "dnsb_couette_norm_noalloc": (c_int, [c_void_p, c_int, c_int, c_int, c_double,
                                          c_void_p, c_void_p]),
    "dnsb_banded_solve": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_int,
                                  c_int, c_int, c_int, c_void_p, c_void_p]),
    # slab decomposition
    "dnsb_periodic_create_slab": (c_int, [C.POINTER(PeriodicDesc), c_int, c_int,
                                          C.POINTER(c_void_p)]),
    "dnsb_periodic_slab_buffers": (c_int, [c_void_p, C.POINTER(c_void_p), C.POINTER(c_void_p)]),
    "dnsb_periodic_slab_connect": (c_int, [c_void_p, C.POINTER(c_void_p), C.POINTER(c_void_p)]),
    "dnsb_periodic_rhs_phase": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_void_p]),
    "dnsb_couette_create_slab": (c_int, [C.POINTER(CouetteDesc), c_int, c_int,
                                         C.POINTER(c_void_p)]),
    "dnsb_couette_slab_buffers": (c_int, [c_void_p, C.POINTER(c_void_p), C.POINTER(c_void_p)]),
    "dnsb_couette_slab_connect": (c_int, [c_void_p, C.POINTER(c_void_p), C.POINTER(c_void_p)]),
    "dnsb_couette_rhs_phase": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_void_p]),
    "dnsb_ipc_handle": (c_int, [c_void_p, c_void_p]),
    "dnsb_ipc_open": (c_int, [c_void_p, C.POINTER(c_void_p)]),
    "dnsb_ipc_close": (c_int, [c_void_p]),
}


class DnsbError(RuntimeError):
    pass


def load(path: Path | str = LIB_PATH):
    """Load the library and declare its signatures (no CUDA call is made)."""
    global _lib
    if _lib is not None and path == LIB_PATH:
        return _lib
    p = Path(path)
    if not p.exists():
        raise DnsbError(
            f"{p} not found: build it with `python -m dnsjax_b200.build` "
            "(this package has no CPU fallback)")
    h = C.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(h, name)
        fn.restype = res
        fn.argtypes = args
    if path == LIB_PATH:
        _lib = h
    return h


def lib():
    """The loaded library, after checking that a CUDA device is usable."""
    import torch

    if not torch.cuda.is_available():
        raise DnsbError("dnsjax_b200 needs a CUDA device (no CPU fallback)")
    return load()


def check(rc: int) -> None:
    if rc != 0:
        msg = _lib.dnsb_last_error().decode() if _lib is not None else ""
        raise DnsbError(f"libdnsb error {rc}: {msg}")


def launch_count() -> int:
    return int(load().dnsb_launch_count())


def ptr(t) -> int:
    """Device address of a contiguous torch tensor."""
    if t is None:
        return None
    if not t.is_contiguous():
        raise DnsbError("tensor must be contiguous")
    if not t.is_cuda:
        raise DnsbError("tensor must live on the GPU")
    return t.data_ptr()


def stream_handle(stream=None) -> int:
    import torch

    s = torch.cuda.current_stream() if stream is None else stream
    return s.cuda_stream


def as_c(arr, ctype=C.c_double):
    """Host pointer of a C-contiguous numpy array (keep `arr` alive)."""
    return arr.ctypes.data_as(C.POINTER(ctype))
