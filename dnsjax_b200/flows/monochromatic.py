"""Triply-periodic flows on the GPU (Kolmogorov, Waleffe, decaying box).

Mirrors src/dnsjax/flows/monochromatic.py.  ``TriplyPeriodicFlow`` holds
the host-side setup -- base flow and its curl / self-interaction on the
padded y grid (:116-208), forcing data (:210-267), the Crank-Nicolson
coefficients ``ldt_1``, ``ildt_2`` with the mean mode zeroed (:269-285) --
and a ``dnsb_periodic`` context.  Its methods are the stepper callables
(``get_rhs``, ``predict``, ``correct``, ``norm``), ``correct_velocity``
(divergence correction + mean-mode zeroing, :516-565), ``get_stats``
(E, I, D, E', :433-510), ``init_state`` and the 3D transforms.  Tensors are
complex128 in the ``(3, ny-1, nz-1, nx//2)`` ``[ky, kz, kx]`` layout.
"""

from __future__ import annotations

import numpy as np

from .. import _lib
from ..geometries.triply_periodic import Fourier
from ..parameters import Parameters, derive, monochromatic_systems, padded_sizes
from ..timestep import StepGraph, make_fused_stepper, make_stepper


class TriplyPeriodicFlow:
    """``slab=(nranks, rank)`` makes this flow one rank's share of a slab
    decomposition (see dnsjax_b200.slab): its tensors hold the kx modes
    [rank nx/2/nranks, (rank+1) nx/2/nranks), as the reference's kx-sharded
    arrays do (sharding.py:107-129)."""

    def __init__(self, p: Parameters, ly: float | None = None,
                 slab: tuple[int, int] | None = None):
        import torch

        L = _lib.lib()
        self.params = p
        d = derive(p)
        self.derived = d
        if ly is not None:
            d.ly = ly
        self.ly = float(d.ly)
        r = p.res
        # res.double_precision = False (parameters.py:63 of the reference)
        # selects the mixed form: the RHS transforms and product in FP32,
        # the state, the curl, the projection, the corrector and the norms in
        # FP64.
        self.rhs_fp32 = r.double_precision is False
        self.system = p.phys.system
        self.nx, self.ny, self.nz = r.nx, r.ny, r.nz
        self.nx_p, self.ny_p, self.nz_p = padded_sizes(p)
        self.re = p.phys.re
        self.dt = p.step.dt
        self.c = p.step.implicitness
        self.fourier = f = Fourier.build(r.nx, r.ny, r.nz, p.geo.lx, self.ly, p.geo.lz)
        self.nranks, self.rank = (0, 0) if slab is None else (int(slab[0]), int(slab[1]))
        nkx = r.nx // 2 // max(self.nranks, 1)
        self.kx_range = (self.rank * nkx, (self.rank + 1) * nkx)
        self.spec_shape = (3, r.ny - 1, r.nz - 1, nkx)
        self.kx_axis = 3
        self.phys_shape = (3, self.ny_p, self.nz_p, self.nx_p)
        self._setup_base_flow(d)

        ldt_1 = 1 / self.dt + (1 - self.c) * f.lapl / self.re
        ildt_2 = 1 / (1 / self.dt - self.c * f.lapl / self.re)
        ldt_1 = np.array(ldt_1, dtype=np.float64)
        ildt_2 = np.array(ildt_2, dtype=np.float64)
        ldt_1[0, 0, 0] = 0.0
        ildt_2[0, 0, 0] = 0.0
        self.ldt_1, self.ildt_2 = ldt_1, ildt_2

        f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64)  # noqa: E731
        hold = dict(kx=f64(f.kx.reshape(-1)), ky=f64(f.ky.reshape(-1)),
                    kz=f64(f.kz.reshape(-1)), U=f64(self.base_flow),
                    cU=f64(self.curl_base_flow), nU=f64(self.nonlin_base_flow),
                    l1=f64(ldt_1), l2=f64(ildt_2))
        c_d = _lib.as_c
        desc = _lib.PeriodicDesc(
            r.nx, r.ny, r.nz, self.nx_p, self.ny_p, self.nz_p, self.dt, self.c,
            c_d(hold["kx"]), c_d(hold["ky"]), c_d(hold["kz"]),
            c_d(hold["U"]), c_d(hold["cU"]), c_d(hold["nU"]),
            c_d(hold["l1"]), c_d(hold["l2"]))
        h = _lib.C.c_void_p()
        if self.nranks:
            _lib.check(L.dnsb_periodic_create_slab(_lib.C.byref(desc), self.nranks, self.rank,
                                                   _lib.C.byref(h)))
        else:
            _lib.check(L.dnsb_periodic_create(_lib.C.byref(desc), _lib.C.byref(h)))
        self._ctx = h
        self._L = L
        if self.rhs_fp32:
            _lib.check(L.dnsb_periodic_set_rhs_precision(self._ctx, 1))
        self._scratch = torch.empty(2, dtype=torch.float64, device="cuda")

    def _setup_base_flow(self, d) -> None:
        """Base flow U(y) on the padded grid (monochromatic.py:116-208)."""
        nyp = self.ny_p
        bfc = np.zeros(nyp // 2 + 1, dtype=np.complex128)
        self.qf = 1
        if self.system in monochromatic_systems:
            if self.system == "kolmogorov":
                bfc[self.qf] += -0.5j   # sin(2 pi y / Ly)
            else:
                bfc[self.qf] += 0.5     # cos(2 pi y / Ly)
            self.force_amplitude = np.pi**2 / (4 * self.re)
            self.ekin_lam = 1.0 / 4.0
            self.input_lam = np.pi**2 / (8 * self.re)
            self.dissip_lam = self.input_lam
        elif self.system == "decaying-box":
            self.force_amplitude = 0.0
            self.ekin_lam = self.input_lam = self.dissip_lam = 0.0
        else:
            raise NotImplementedError(self.system)
        dbfc = 1j * (2 * np.pi / self.ly) * bfc
        U = np.zeros((3, nyp))
        dU = np.zeros((3, nyp))
        cU = np.zeros((3, nyp))
        nU = np.zeros((3, nyp))
        U[0] = np.fft.irfft(bfc, n=nyp, norm="forward")
        dU[0] = np.fft.irfft(dbfc, n=nyp, norm="forward")
        cU[2] = -dU[0]
        nU[1] = U[0] * dU[0]
        th = d.tilt_rad
        if abs(th) != 0:
            U[2] = np.sin(th) * U[0]
            U[0] = U[0] * np.cos(th)
            dU[2] = np.sin(th) * dU[0]
            dU[0] = dU[0] * np.cos(th)
            cU[0] = -np.sin(th) * cU[2]
            cU[2] = cU[2] * np.cos(th)
        self.base_flow, self.curl_base_flow, self.nonlin_base_flow = U, cU, nU
        if self.system in monochromatic_systems:
            qf = self.qf
            c, s = np.cos(th), np.sin(th)
            if not d.tilt:
                self.forced_modes = ((0, 0), (qf, -qf), (0, 0), (0, 0))
            elif d.tilt_90:
                self.forced_modes = ((2, 2), (qf, -qf), (0, 0), (0, 0))
            else:
                self.forced_modes = ((0, 0, 2, 2), (qf, -qf, qf, -qf),
                                     (0, 0, 0, 0), (0, 0, 0, 0))
            if not d.tilt or d.tilt_90:
                self.unit_force = (np.array([-0.5j, 0.5j])
                                   if self.system == "kolmogorov"
                                   else np.array([0.5, 0.5], dtype=complex))
            elif self.system == "kolmogorov":
                self.unit_force = np.array([-0.5j * c, 0.5j * c, -0.5j * s, 0.5j * s])
            else:
                self.unit_force = np.array([0.5 * c, 0.5 * c, -0.5j * s, 0.5j * s])

    def __del__(self):
        ctx = getattr(self, "_ctx", None)
        if ctx is not None and ctx.value:
            self._L.dnsb_periodic_destroy(ctx)
            self._ctx = None

    # -- helpers ---------------------------------------------------------------
    def _new(self):
        import torch

        return torch.empty(self.spec_shape, dtype=torch.complex128, device="cuda")

    def _check(self, t):
        if tuple(t.shape) != self.spec_shape:
            raise ValueError(f"expected shape {self.spec_shape}, got {tuple(t.shape)}")
        if str(t.dtype) != "torch.complex128":
            raise ValueError("expected complex128")
        return _lib.ptr(t)

    # -- stepper callables (monochromatic.py:366-410) ----------------------------
    def get_rhs(self, state, out=None):
        out = self._new() if out is None else out
        _lib.check(self._L.dnsb_periodic_rhs(
            self._ctx, self._check(state), self._check(out), _lib.stream_handle()))
        return out

    # -- slab decomposition (dnsjax_b200.slab) -----------------------------------
    def slab_buffers(self):
        """This rank's receive buffers (device pointers): the padded-z share
        the z inverse fills, and the pass buffer the x pass fills."""
        bx, bk = _lib.C.c_void_p(), _lib.C.c_void_p()
        _lib.check(self._L.dnsb_periodic_slab_buffers(self._ctx, _lib.C.byref(bx),
                                                      _lib.C.byref(bk)))
        return bx.value, bk.value

    def slab_connect(self, bx, bk) -> None:
        """Every rank's receive buffers, as this process addresses them."""
        arr = _lib.C.c_void_p * len(bx)
        _lib.check(self._L.dnsb_periodic_slab_connect(self._ctx, arr(*bx), arr(*bk)))

    def rhs_phase(self, state, out, phase: int):
        _lib.check(self._L.dnsb_periodic_rhs_phase(
            self._ctx, self._check(state), self._check(out), int(phase),
            _lib.stream_handle()))
        return out

    def predict(self, state, rhs, out=None):
        out = self._new() if out is None else out
        _lib.check(self._L.dnsb_periodic_predict(
            self._ctx, self._check(state), self._check(rhs), self._check(out),
            _lib.stream_handle()))
        return out

    def correct(self, state_prev, prediction, rhs_prev, rhs_next):
        """Incremental CN corrector -> (prediction_new, correction)."""
        out, corr = self._new(), self._new()
        _lib.check(self._L.dnsb_periodic_correct(
            self._ctx, self._check(prediction), self._check(rhs_prev),
            self._check(rhs_next), self._check(out), self._check(corr), None,
            _lib.stream_handle()))
        return out, corr

    def correct_fused(self, state_prev, prediction, rhs_prev, rhs_next, err,
                      out=None):
        out = self._new() if out is None else out
        _lib.check(self._L.dnsb_periodic_correct(
            self._ctx, self._check(prediction), self._check(rhs_prev),
            self._check(rhs_next), self._check(out), None, _lib.ptr(err),
            _lib.stream_handle()))
        return out

    def norm(self, v, out=None):
        import torch

        out = torch.empty(1, dtype=torch.float64, device="cuda") if out is None else out
        _lib.check(self._L.dnsb_periodic_norm(self._ctx, self._check(v),
                                              _lib.ptr(out), _lib.stream_handle()))
        return out

    def correct_velocity(self, state, divergence: bool | None = None):
        """Divergence correction, then mean mode := 0; returns (state, None)."""
        if divergence is None:
            dbg = self.params.debug
            divergence = True if dbg is None else dbg.correct_divergence
        _lib.check(self._L.dnsb_periodic_correct_velocity(
            self._ctx, self._check(state), self._check(state), int(divergence),
            _lib.stream_handle()))
        return state, None

    def set_rhs_precision(self, fp32: bool, compensated: bool = False) -> None:
        """FP32 (True) or FP64 (False) RHS passes for the following RHS calls
        (the ``res.double_precision`` switch); with ``compensated`` the FP32
        passes' register DFTs carry two-sum compensated accumulation."""
        mode = (2 if compensated else 1) if fp32 else 0
        _lib.check(self._L.dnsb_periodic_set_rhs_precision(self._ctx, mode))
        self.rhs_fp32 = bool(fp32)

    def set_graph_unroll(self, n: int) -> None:
        """Corrector iterations that step graphs made afterwards hold as
        straight-line kernels ahead of the device-controlled loop (see
        dnsb_periodic_set_graph_unroll); the states are the same bit for
        bit."""
        _lib.check(self._L.dnsb_periodic_set_graph_unroll(self._ctx, int(n)))
        self._graph_unroll = int(n)

    def make_step_graph(self, state, tol: float | None = None,
                        max_iter: int | None = None, divergence: bool | None = None,
                        unroll: int | None = None):
        """A CUDA graph of one full time step bound to `state` (updated in
        place by every launch); see StepGraph.  ``unroll``: corrector
        iterations held as straight-line kernels (set_graph_unroll)."""
        st = self.params.step
        if divergence is None:
            dbg = self.params.debug
            divergence = True if dbg is None else dbg.correct_divergence
        tol = st.corrector_tolerance if tol is None else tol
        max_iter = st.max_corrector_iterations if max_iter is None else max_iter

        def make():
            return StepGraph(self._L, state, lambda h: self._L.dnsb_periodic_step_graph_create(
                self._ctx, self._check(state), float(tol), int(max_iter), int(divergence), h))

        if unroll is None:
            return make()
        prev = getattr(self, "_graph_unroll", 0)
        self.set_graph_unroll(unroll)
        try:
            return make()
        finally:
            self.set_graph_unroll(prev)

    # -- variants of the passes (no counterpart in the reference) ----------------
    def autotune(self, state, reps: int = 5) -> dict:
        """Times every kernel variant of each pass (and, for Couette, the
        IMM) on this flow's sizes from `state` and keeps the fastest (see
        dnsb_periodic_autotune); returns the choices and the mean times."""
        n = 5
        chosen = (_lib.C.c_int * n)()
        ms = (_lib.C.c_float * (3 * n))()
        _lib.check(self._L.dnsb_periodic_autotune(self._ctx, self._check(state), int(reps),
                                                 chosen, ms, _lib.stream_handle()))
        return {"variants": list(chosen), "ms": [list(ms[3 * k:3 * k + 3]) for k in range(n)],
                 "stages": ["y inverse", "z inverse", "x", "z forward", "y forward"]}

    def set_variants(self, variants) -> None:
        arr = (_lib.C.c_int * 5)(*[int(v) for v in variants])
        _lib.check(self._L.dnsb_periodic_set_variants(self._ctx, arr))

    def get_stats(self, state) -> dict:
        """E, I, D, E' (monochromatic.py:433-505)."""
        return self.stats_from_sums(self.stats_sums(state))

    def stats_sums(self, state):
        """The sums get_stats needs, over this flow's modes (a slab rank's
        share; the shares add up over the ranks): sum k_metric |u|^2, the
        enstrophy sum, and the forcing's projection on the forced modes this
        flow holds."""
        _lib.check(self._L.dnsb_periodic_energy_sums(
            self._ctx, self._check(state), _lib.ptr(self._scratch),
            _lib.stream_handle()))
        norm2, ens_sum = (float(v) for v in self._scratch.tolist())
        proj = 0.0
        if self.system in monochromatic_systems:
            k0, k1 = self.kx_range
            c, iy, iz, ix = (np.array(i) for i in self.forced_modes)
            mine = (ix >= k0) & (ix < k1)
            if mine.any():
                vals = state[(c[mine], iy[mine], iz[mine], ix[mine] - k0)].cpu().numpy()
                proj = float(np.sum(np.conj(self.unit_force[mine] * self.force_amplitude)
                                    * vals).real)
        return norm2, ens_sum, proj

    def stats_from_sums(self, sums) -> dict:
        norm2, ens_sum, proj = sums
        ep = norm2 / 2
        re = self.re
        if self.system in monochromatic_systems:
            inp = proj + self.input_lam
            energy = ep - self.ekin_lam + inp / self.force_amplitude
        else:
            # The reference reads flow.unit_force here, which only forced
            # systems define; for the decaying box the input is zero.
            inp = self.input_lam
            energy = ep
        enstrophy = ens_sum + 2 * inp * re - self.input_lam * re
        return {"E": energy, "I": inp, "D": enstrophy / re, "E'": ep}

    # -- transforms (operators.py:59-101) -----------------------------------------
    def spec_to_phys(self, spec):
        import torch

        out = torch.empty(self.phys_shape, dtype=torch.float64, device="cuda")
        _lib.check(self._L.dnsb_periodic_spec_to_phys(
            self._ctx, self._check(spec), _lib.ptr(out), _lib.stream_handle()))
        return out

    def phys_to_spec(self, phys):
        out = self._new()
        _lib.check(self._L.dnsb_periodic_phys_to_spec(
            self._ctx, _lib.ptr(phys.contiguous()), self._check(out),
            _lib.stream_handle()))
        return out

    def init_state(self, snapshot=None):
        """monochromatic.py:294-314: laminar (zeros) or an npz snapshot's
        ``velocity_phys`` minus the base flow."""
        import torch

        if self.params.init.start_from_laminar or snapshot is None:
            return torch.zeros(self.spec_shape, dtype=torch.complex128, device="cuda")
        arr = np.load(snapshot)["velocity_phys"].astype(np.float64)
        arr = arr - self.base_flow[:, :, None, None]
        return self.phys_to_spec(torch.as_tensor(np.ascontiguousarray(arr),
                                                 device="cuda"))

    def save_snapshot(self, path, state) -> None:
        """Write ``state`` as an npz snapshot the reference's init_state
        reads (monochromatic.py:302-311): ``velocity_phys`` = the physical
        perturbation velocity plus the base flow."""
        phys = self.spec_to_phys(state).cpu().numpy()
        np.savez(path, velocity_phys=phys + self.base_flow[:, :, None, None])

    def make_stepper(self, fused: bool = True):
        if fused:
            return make_fused_stepper(self)
        return make_stepper(
            lambda s: self.get_rhs(s),
            lambda s, r: self.predict(s, r),
            lambda sp, pr, rp, rn: self.correct(sp, pr, rp, rn),
            lambda cr: self.norm(cr))


# -- module-level interface bound to the global params --------------------------
flow: TriplyPeriodicFlow | None = None
_steppers = None


def _flow() -> TriplyPeriodicFlow:
    global flow, _steppers
    if flow is None:
        from ..parameters import derived_params, params

        flow = TriplyPeriodicFlow(params, ly=derived_params.ly)
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
