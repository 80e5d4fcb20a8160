"""Triply-periodic flows (Kolmogorov / Waleffe / decaying box), NumPy FP64.

Oracle restatement (test infrastructure only) of
``src/dnsjax/geometries/triply_periodic.py`` and
``src/dnsjax/flows/monochromatic.py``.  Spectral layout ``(3, ny-1, nz-1,
nx//2)`` in ``[ky, kz, kx]`` order; physical ``(3, My, Mz, Mx)``.
"""

from __future__ import annotations

import numpy as np

from .config import MONOCHROMATIC, Config
from .fft import (
    complex_harmonics,
    get_nonlin,
    phys_to_spec,
    real_harmonics,
    spec_to_phys,
)


class PeriodicSetup:
    """Wavenumbers (triply_periodic.py:14-75) and flow data
    (monochromatic.py:85-285)."""

    def __init__(self, cfg: Config) -> None:
        self.cfg = cfg
        two_pi = 2 * np.pi
        self.kx = (real_harmonics(cfg.nx).reshape(1, 1, -1) * two_pi / cfg.lx)
        self.kz = complex_harmonics(cfg.nz).reshape(1, -1, 1) * two_pi / cfg.lz
        self.ky = complex_harmonics(cfg.ny).reshape(-1, 1, 1) * two_pi / cfg.ly
        self.k_metric = np.where(self.kx == 0, 1, 2)
        self.lapl = -(self.kx**2 + self.ky**2 + self.kz**2)
        with np.errstate(divide="ignore"):
            self.inv_lapl = np.where(self.lapl < 0, 1 / self.lapl, 0)

        ny_p = cfg.ny_padded
        bfc = np.zeros(ny_p // 2 + 1, dtype=complex)
        self.qf = 1
        if cfg.system in MONOCHROMATIC:
            if cfg.system == "kolmogorov":
                bfc[self.qf] += -0.5j
            else:
                bfc[self.qf] += 0.5
            self.force_amplitude = np.pi**2 / (4 * cfg.re)
            self.ekin_lam = 1.0 / 4.0
            self.input_lam = np.pi**2 / (8 * cfg.re)
            self.dissip_lam = self.input_lam
        else:
            self.force_amplitude = 0.0
            self.ekin_lam = 0.0
            self.input_lam = 0.0
            self.dissip_lam = 0.0
        dbfc = 1j * (two_pi / cfg.ly) * bfc

        U = np.zeros((3, ny_p))
        dU = np.zeros((3, ny_p))
        curlU = np.zeros((3, ny_p))
        nlU = np.zeros((3, ny_p))
        U[0] = np.fft.irfft(bfc, n=ny_p, norm="forward")
        dU[0] = np.fft.irfft(dbfc, n=ny_p, norm="forward")
        curlU[2] = -dU[0]
        nlU[1] = U[0] * dU[0]
        th = cfg.tilt_rad
        if abs(th) != 0:
            U[2] = np.sin(th) * U[0]
            U[0] = U[0] * np.cos(th)
            dU[2] = np.sin(th) * dU[0]
            dU[0] = dU[0] * np.cos(th)
            curlU[0] = -np.sin(th) * curlU[2]
            curlU[2] = curlU[2] * np.cos(th)
        self.base_flow = U[:, :, None, None]
        self.dy_base_flow = dU[:, :, None, None]
        self.curl_base_flow = curlU[:, :, None, None]
        self.nonlin_base_flow = nlU[:, :, None, None]

        # monochromatic.py:210-267 (forced modes, unit forcing)
        if cfg.system in MONOCHROMATIC:
            qf = self.qf
            if not cfg.tilt:
                self.forced_modes = ((0, 0), (qf, -qf), (0, 0), (0, 0))
            elif cfg.tilt_90:
                self.forced_modes = ((2, 2), (qf, -qf), (0, 0), (0, 0))
            else:
                self.forced_modes = (
                    (0, 0, 2, 2),
                    (qf, -qf, qf, -qf),
                    (0, 0, 0, 0),
                    (0, 0, 0, 0),
                )
            c, s = np.cos(th), np.sin(th)
            if not cfg.tilt or cfg.tilt_90:
                if cfg.system == "kolmogorov":
                    self.unit_force = np.array([-0.5j, 0.5j])
                else:
                    self.unit_force = np.array([0.5, 0.5], dtype=complex)
            elif cfg.system == "kolmogorov":
                self.unit_force = np.array(
                    [-0.5j * c, 0.5j * c, -0.5j * s, 0.5j * s]
                )
            else:
                self.unit_force = np.array(
                    [0.5 * c, 0.5 * c, -0.5j * s, 0.5j * s]
                )

        # monochromatic.py:269-285 (CN coefficients, mean mode zeroed)
        ldt_1 = 1 / cfg.dt + (1 - cfg.implicitness) * self.lapl / cfg.re
        ildt_2 = 1 / (1 / cfg.dt - cfg.implicitness * self.lapl / cfg.re)
        ldt_1 = np.array(ldt_1, dtype=float)
        ildt_2 = np.array(ildt_2, dtype=float)
        ldt_1[0, 0, 0] = 0
        ildt_2[0, 0, 0] = 0
        self.ldt_1 = ldt_1
        self.ildt_2 = ildt_2

    # -- spectral operators (triply_periodic.py:104-148) -------------------
    def curl(self, u):
        kx, ky, kz = self.kx, self.ky, self.kz
        return 1j * np.array(
            [ky * u[2] - kz * u[1], kz * u[0] - kx * u[2], kx * u[1] - ky * u[0]]
        )

    def divergence(self, u):
        return 1j * self.kx * u[0] + 1j * self.ky * u[1] + 1j * self.kz * u[2]

    def gradient(self, p):
        return np.array([1j * self.kx * p, 1j * self.ky * p, 1j * self.kz * p])

    # -- stepper callables (monochromatic.py:320-410) ----------------------
    def get_rhs(self, state):
        """monochromatic.py:366-386: NL minus grad(inv_lapl(div NL))."""
        cfg = self.cfg
        nonlin = get_nonlin(
            state,
            self.base_flow,
            self.curl_base_flow,
            self.nonlin_base_flow,
            lambda v: spec_to_phys(v, cfg),
            lambda v: phys_to_spec(v, cfg),
            self.curl,
        )
        lapl_p = self.divergence(nonlin)
        return nonlin - self.gradient(self.inv_lapl * lapl_p)

    def predict(self, state, rhs):
        """monochromatic.py:320-333."""
        return (state * self.ldt_1 + rhs) * self.ildt_2

    def correct(self, state_prev, prediction, rhs_prev, rhs_next):
        """monochromatic.py:336-355 (incremental CN corrector)."""
        corr = self.cfg.implicitness * (rhs_next - rhs_prev) * self.ildt_2
        return prediction + corr, corr

    def norm2(self, v):
        """triply_periodic.py:81-96: Parseval sum, real part."""
        return float(np.sum(np.conj(v) * self.k_metric * v).real)

    def norm(self, v):
        return float(np.sqrt(self.norm2(v)))

    def correct_velocity(self, state, divergence=True):
        """monochromatic.py:516-565: projection then mean mode := 0."""
        out = state
        if divergence:
            out = state + (-self.gradient(self.inv_lapl * self.divergence(state)))
        out = out.copy()
        out[:, 0:1, 0:1, 0:1] = 0
        return out

    # -- stats (monochromatic.py:433-505) -----------------------------------
    def stats(self, state) -> dict:
        ep = self.norm2(state) / 2
        if self.cfg.system in MONOCHROMATIC:
            fm = self.forced_modes
            vals = state[fm]
            inp = float(
                np.sum(np.conj(self.unit_force * self.force_amplitude) * vals).real
            ) + self.input_lam
        else:
            inp = self.input_lam
        re = self.cfg.re
        enstrophy = (
            float(np.sum(-(self.lapl * (np.conj(state) * state))).real)
            + 2 * inp * re
            - self.input_lam * re
        )
        diss = enstrophy / re
        if self.cfg.system in MONOCHROMATIC:
            energy = ep - self.ekin_lam + inp / self.force_amplitude
        else:
            energy = ep
        return {"E": energy, "I": inp, "D": diss, "E'": ep}
