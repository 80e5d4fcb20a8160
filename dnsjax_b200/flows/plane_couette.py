"""Plane Couette flow on the GPU: the reference's flow interface over libdnsb.

Mirrors src/dnsjax/flows/plane_couette.py.  ``PlaneCouetteFlow`` holds the
host-side setup (CGL grid, base flow ``U = y``, FD stencils, IMM operators)
and a ``dnsb_couette`` context; its methods are the four stepper callables
(``get_rhs``, ``predict``, ``correct``, ``norm``), ``correct_velocity``
(the identity, plane_couette.py:575-582), ``get_stats`` (E', :591-613),
``init_state`` and the 2D transforms.  All arithmetic on the state runs in
the CUDA kernels; tensors are complex128 in the ``(3, nz-1, nx//2, ny)``
``[kz, kx, y]`` layout.

Module-level ``predict_and_correct`` / ``iterate_correction`` /
``correct_velocity`` / ``get_stats`` / ``init_state`` act on a flow built
from the global ``params`` on first use, like the reference's import-time
singletons.
"""

from __future__ import annotations

import numpy as np

from .. import _lib
from ..fd import build_diff_matrices, cgl_grid, diff_bands
from ..geometries.cartesian import Fourier, precompute_imm, precompute_imm_gpu, simpson_weights
from ..parameters import Parameters, derive, padded_sizes
from ..timestep import StepGraph, make_fused_stepper, make_stepper


class PlaneCouetteFlow:
    """``slab=(nranks, rank)`` makes this flow one rank's share of a slab
    decomposition (see dnsjax_b200.slab): its tensors and IMM operators hold
    the kx modes [rank nx/2/nranks, (rank+1) nx/2/nranks), as the reference's
    kx-sharded arrays do (sharding.py:107-129); ``imm``, when given, is the
    whole problem's."""

    def __init__(self, p: Parameters, imm: dict | None = None, ly: float | None = None,
                 precompute: str = "gpu", slab: tuple[int, int] | None = None):
        import torch

        L = _lib.lib()
        self.params = p
        d = derive(p)
        self.ly = float(d.ly if ly is None else ly)
        r = p.res
        # res.double_precision = False (parameters.py:63 of the reference)
        # selects the mixed form: the RHS transforms and products in FP32,
        # the state, the IMM (banded LU, 2x2 solve) and the norms in FP64.
        self.rhs_fp32 = p.res.double_precision is False
        self.nx, self.ny, self.nz = r.nx, r.ny, r.nz
        self.nx_p, _, self.nz_p = padded_sizes(p)
        self.p = r.fd_order
        self.dt = p.step.dt
        self.c = p.step.implicitness
        self.nu = 1.0 / p.phys.re
        self.fourier = Fourier.build(r.nx, r.nz, p.geo.lx, p.geo.lz)
        self.ys = cgl_grid(r.ny)
        self.D1, self.D2 = build_diff_matrices(self.ys, self.p)
        j01, w1, j02, w2 = diff_bands(self.ys, self.p)
        ny = r.ny
        U = np.zeros((3, ny))
        U[0] = self.ys
        cU = np.zeros((3, ny))
        cU[2] = -1.0
        nU = np.zeros((3, ny))
        nU[1] = self.ys * 1.0
        self.base_flow, self.curl_base_flow, self.nonlin_base_flow = U, cU, nU
        self.nranks, self.rank = (0, 0) if slab is None else (int(slab[0]), int(slab[1]))
        nkx = r.nx // 2 // max(self.nranks, 1)
        self.kx_range = k0, k1 = (self.rank * nkx, (self.rank + 1) * nkx)
        kx_local = self.fourier.kx_global[k0:k1]
        self.spec_shape = (3, r.nz - 1, nkx, ny)
        self.kx_axis = 2
        self.phys_shape = (3, ny, self.nz_p, self.nx_p)
        self.simpson = simpson_weights(self.ys)

        f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64)  # noqa: E731
        i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)  # noqa: E731
        # host arrays stay referenced by `hold` until create() has copied them
        hold = dict(kx=f64(self.fourier.kx_global), kz=f64(self.fourier.kz_global),
                    ys=f64(self.ys), j01=i32(j01), w1=f64(w1), j02=i32(j02),
                    w2=f64(w2), U=f64(U), cU=f64(cU), nU=f64(nU))
        c_d = _lib.as_c
        desc = _lib.CouetteDesc(
            r.nx, ny, r.nz, self.nx_p, self.nz_p, self.p,
            self.dt, self.c, self.nu, self.ly,
            c_d(hold["kx"]), c_d(hold["kz"]), c_d(hold["ys"]),
            c_d(hold["j01"], _lib.C.c_int), c_d(hold["w1"]),
            c_d(hold["j02"], _lib.C.c_int), c_d(hold["w2"]),
            c_d(hold["U"]), c_d(hold["cU"]), c_d(hold["nU"]))
        h = _lib.C.c_void_p()
        if self.nranks:
            _lib.check(L.dnsb_couette_create_slab(_lib.C.byref(desc), self.nranks, self.rank,
                                                  _lib.C.byref(h)))
        else:
            _lib.check(L.dnsb_couette_create(_lib.C.byref(desc), _lib.C.byref(h)))
        self._ctx = h
        self._L = L
        if self.rhs_fp32:
            _lib.check(L.dnsb_couette_set_rhs_precision(self._ctx, 1))

        # Influence-matrix data (cartesian.py:575-801): given, or computed
        # once here -- on the GPU ("gpu") or on the host as the reference
        # does ("host").
        # A slab rank computes (or takes) the operators of its kx modes only.
        if imm is None:
            if precompute == "gpu":
                imm = precompute_imm_gpu(kx_local, self.fourier.kz_global,
                                         self.p, self.dt, self.c, self.nu, self.D1, self.D2)
            elif precompute == "host":
                imm = precompute_imm(self.ys, kx_local,
                                     self.fourier.kz_global, self.p, self.dt,
                                     self.c, self.nu, self.D1, self.D2)
            else:
                raise ValueError(f"precompute must be 'gpu' or 'host', got {precompute!r}")
        elif self.nranks:
            imm = {k: v[:, k0:k1] for k, v in imm.items()}

        def to_dev(a, dt_np, dt_t):
            if isinstance(a, torch.Tensor):
                return a.to(device="cuda", dtype=dt_t).contiguous()
            return torch.as_tensor(np.ascontiguousarray(a, dt_np), device="cuda")

        dev = {}
        for k in ("Lk_ab", "Hk_ab", "v1", "v2", "q1", "q2", "M_inv", "p1", "p2"):
            dev[k] = to_dev(imm[k], np.float64, torch.float64)
        for k in ("Lk_piv", "Hk_piv"):
            dev[k] = to_dev(imm[k], np.int32, torch.int32)
        self.imm = dev
        ops = _lib.ImmOps(*[_lib.ptr(dev[k]) for k in (
            "Lk_ab", "Lk_piv", "Hk_ab", "Hk_piv", "v1", "v2", "q1", "q2", "M_inv")])
        _lib.check(L.dnsb_couette_bind_imm(self._ctx, _lib.C.byref(ops)))
        self._scratch = torch.empty(2, dtype=torch.float64, device="cuda")

    def __del__(self):
        ctx = getattr(self, "_ctx", None)
        if ctx is not None and ctx.value:
            self._L.dnsb_couette_destroy(ctx)
            self._ctx = None

    # -- helpers ------------------------------------------------------------
    def _new(self):
        import torch

        return torch.empty(self.spec_shape, dtype=torch.complex128, device="cuda")

    def _check(self, t):
        if tuple(t.shape) != self.spec_shape:
            raise ValueError(f"expected shape {self.spec_shape}, got {tuple(t.shape)}")
        if str(t.dtype) != "torch.complex128":
            raise ValueError("expected complex128")
        return _lib.ptr(t)

    # -- stepper callables (plane_couette.py:274-549) -------------------------
    def get_rhs(self, state, out=None):
        out = self._new() if out is None else out
        _lib.check(self._L.dnsb_couette_rhs(
            self._ctx, self._check(state), self._check(out), _lib.stream_handle()))
        return out

    # -- slab decomposition (dnsjax_b200.slab) -----------------------------------
    def slab_buffers(self):
        """This rank's receive buffers (device pointers): the padded-z share
        the z inverse fills, and the pass buffer the x pass fills."""
        bx, bk = _lib.C.c_void_p(), _lib.C.c_void_p()
        _lib.check(self._L.dnsb_couette_slab_buffers(self._ctx, _lib.C.byref(bx),
                                                     _lib.C.byref(bk)))
        return bx.value, bk.value

    def slab_connect(self, bx, bk) -> None:
        """Every rank's receive buffers, as this process addresses them."""
        arr = _lib.C.c_void_p * len(bx)
        _lib.check(self._L.dnsb_couette_slab_connect(self._ctx, arr(*bx), arr(*bk)))

    def rhs_phase(self, state, out, phase: int):
        _lib.check(self._L.dnsb_couette_rhs_phase(
            self._ctx, self._check(state), self._check(out), int(phase),
            _lib.stream_handle()))
        return out

    def imm_iteration(self, vel_n, vel_j, nl_n, nl_j, out=None, corr=None,
                      err=None):
        out = self._new() if out is None else out
        _lib.check(self._L.dnsb_couette_imm(
            self._ctx, self._check(vel_n), self._check(vel_j), self._check(nl_n),
            self._check(nl_j), self._check(out),
            None if corr is None else self._check(corr),
            None if err is None else _lib.ptr(err), _lib.stream_handle()))
        return out

    def predict(self, state, rhs):
        """plane_couette.py:507-519: IMM with (u^n, u^n, N^n, N^n)."""
        return self.imm_iteration(state, state, rhs, rhs)

    def correct(self, state_prev, prediction, rhs_prev, rhs_next):
        """plane_couette.py:522-540 -> (prediction_new, correction)."""
        corr = self._new()
        new = self.imm_iteration(state_prev, prediction, rhs_prev, rhs_next,
                                 corr=corr)
        return new, corr

    def correct_fused(self, state_prev, prediction, rhs_prev, rhs_next, err,
                      out=None):
        """``correct`` + ``norm`` in one kernel; the correction itself is not
        stored.  ``out`` may be ``prediction`` (it is donated)."""
        return self.imm_iteration(state_prev, prediction, rhs_prev, rhs_next,
                                  out=out, err=err)

    def norm(self, v, out=None):
        """plane_couette.py:543-549 (Simpson in y, / ly), device scalar."""
        import torch

        out = torch.empty(1, dtype=torch.float64, device="cuda") if out is None else out
        _lib.check(self._L.dnsb_couette_norm(self._ctx, self._check(v),
                                             _lib.ptr(out), _lib.stream_handle()))
        return out

    def set_rhs_precision(self, fp32: bool, compensated: bool = False) -> None:
        """FP32 (True) or FP64 (False) RHS passes for the following RHS calls
        (the ``res.double_precision`` switch, applied per call); with
        ``compensated`` the FP32 passes' register DFTs carry two-sum
        compensated accumulation."""
        mode = (2 if compensated else 1) if fp32 else 0
        if mode != getattr(self, "_rhs_mode", 1 if self.rhs_fp32 else 0):
            _lib.check(self._L.dnsb_couette_set_rhs_precision(self._ctx, mode))
            self._rhs_mode = mode
            self.rhs_fp32 = bool(fp32)

    def correct_velocity(self, state):
        """plane_couette.py:575-582: pass-through."""
        return state, None

    def set_graph_unroll(self, n: int) -> None:
        """Corrector iterations that step graphs made afterwards hold as
        straight-line kernels ahead of the device-controlled loop (see
        dnsb_couette_set_graph_unroll); the states are the same bit for bit,
        the iterations within the unrolled count enter no conditional node."""
        _lib.check(self._L.dnsb_couette_set_graph_unroll(self._ctx, int(n)))
        self._graph_unroll = int(n)

    def _with_unroll(self, unroll, make):
        """make() with the graph unroll set to `unroll` (None: the current
        setting), the setting restored afterwards."""
        if unroll is None:
            return make()
        prev = getattr(self, "_graph_unroll", 0)
        self.set_graph_unroll(unroll)
        try:
            return make()
        finally:
            self.set_graph_unroll(prev)

    def make_step_graph(self, state, tol: float | None = None,
                        max_iter: int | None = None, unroll: int | None = None):
        """A CUDA graph of one full time step bound to `state` (updated in
        place by every launch); see StepGraph.  ``unroll``: corrector
        iterations held as straight-line kernels (set_graph_unroll)."""
        st = self.params.step
        tol = st.corrector_tolerance if tol is None else tol
        max_iter = st.max_corrector_iterations if max_iter is None else max_iter
        return self._with_unroll(unroll, lambda: StepGraph(
            self._L, state, lambda h: self._L.dnsb_couette_step_graph_create(
                self._ctx, self._check(state), float(tol), int(max_iter), h)))

    # -- variants of the passes (no counterpart in the reference) ----------------
    def autotune(self, state, reps: int = 5) -> dict:
        """Times every kernel variant of each pass (and, for Couette, the
        IMM) on this flow's sizes from `state` and keeps the fastest (see
        dnsb_couette_autotune); returns the choices and the mean times."""
        n = 4
        chosen = (_lib.C.c_int * n)()
        ms = (_lib.C.c_float * (3 * n))()
        _lib.check(self._L.dnsb_couette_autotune(self._ctx, self._check(state), int(reps),
                                                 chosen, ms, _lib.stream_handle()))
        return {"variants": list(chosen), "ms": [list(ms[3 * k:3 * k + 3]) for k in range(n)],
                 "stages": ["z inverse", "x", "z forward", "IMM"]}

    def set_variants(self, variants) -> None:
        arr = (_lib.C.c_int * 4)(*[int(v) for v in variants])
        _lib.check(self._L.dnsb_couette_set_variants(self._ctx, arr))

    def get_stats(self, state) -> dict:
        """plane_couette.py:591-613: E' = ||u||^2 / 2."""
        return self.stats_from_sums(self.stats_sums(state))

    def stats_sums(self, state):
        """||u||^2 over this flow's modes (a slab rank's share)."""
        _lib.check(self._L.dnsb_couette_norm2(
            self._ctx, self._check(state), _lib.ptr(self._scratch),
            _lib.stream_handle()))
        return (float(self._scratch[0].item()),)

    def stats_from_sums(self, sums) -> dict:
        return {"E'": sums[0] / 2}

    def check_status(self):
        """Raises if a bound operator holds an out-of-range pivot or an IMM
        substitution wait gave up since the status was last cleared."""
        _lib.check(self._L.dnsb_couette_check(self._ctx, _lib.stream_handle()))

    def clear_status(self):
        _lib.check(self._L.dnsb_couette_clear_status(self._ctx, _lib.stream_handle()))

    def set_wait_limit(self, polls: int):
        """Polls of a substitution ring slot before the wait gives up."""
        _lib.check(self._L.dnsb_couette_set_wait_limit(self._ctx, int(polls)))

    # -- transforms (operators.py:104-146) -------------------------------------
    def spec_to_phys(self, spec):
        import torch

        out = torch.empty(self.phys_shape, dtype=torch.float64, device="cuda")
        _lib.check(self._L.dnsb_couette_spec_to_phys(
            self._ctx, self._check(spec), _lib.ptr(out), _lib.stream_handle()))
        return out

    def phys_to_spec(self, phys):
        out = self._new()
        _lib.check(self._L.dnsb_couette_phys_to_spec(
            self._ctx, _lib.ptr(phys.contiguous()), self._check(out),
            _lib.stream_handle()))
        return out

    def init_state(self, snapshot=None):
        """plane_couette.py:225-248: laminar (zeros) or an npz snapshot's
        ``velocity_phys_nonexpanded``."""
        import torch

        if self.params.init.start_from_laminar or snapshot is None:
            return torch.zeros(self.spec_shape, dtype=torch.complex128, device="cuda")
        arr = np.load(snapshot)["velocity_phys_nonexpanded"].astype(np.float64)
        return self.phys_to_spec(torch.as_tensor(arr, device="cuda"))

    def save_snapshot(self, path, state) -> None:
        """Write ``state`` as an npz snapshot the reference's init_state
        reads (plane_couette.py:233-242): ``velocity_phys_nonexpanded`` =
        the physical perturbation velocity (no base flow)."""
        np.savez(path, velocity_phys_nonexpanded=self.spec_to_phys(state).cpu().numpy())

    # -- stepper ---------------------------------------------------------------
    def make_stepper(self, fused: bool = True):
        if fused:
            return make_fused_stepper(self)
        return make_stepper(
            lambda s: self.get_rhs(s),
            lambda s, r: self.predict(s, r),
            lambda sp, pr, rp, rn: self.correct(sp, pr, rp, rn),
            lambda cr: self.norm(cr))


# -- module-level interface bound to the global params -------------------------
flow: PlaneCouetteFlow | None = None
_steppers = None


def _flow() -> PlaneCouetteFlow:
    global flow, _steppers
    if flow is None:
        from ..parameters import params

        flow = PlaneCouetteFlow(params)
        _steppers = flow.make_stepper(fused=True)
    return flow


def predict_and_correct(state):
    _flow()
    return _steppers[0](state)


def iterate_correction(state_prev, prediction, rhs_prev):
    _flow()
    return _steppers[1](state_prev, prediction, rhs_prev)


def correct_velocity(state):
    return _flow().correct_velocity(state)


def get_stats(state) -> dict:
    return _flow().get_stats(state)


def init_state(snapshot=None):
    return _flow().init_state(snapshot)


def save_snapshot(path, state) -> None:
    _flow().save_snapshot(path, state)
