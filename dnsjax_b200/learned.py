"""Learned corrector guess for plane Couette.

A per-(kz, kx)-mode MLP, 1.19M parameters at 128x129x128 (12 Ny + 2 ->
``hidden`` = 512 -> 6 Ny), with BF16 weights and activations and FP32
accumulation on the tensor cores (``dnsb_mlp_*``, ``csrc/learned.cu``).
For every mode it guesses the converged corrector correction u^{n+1} - u_p
(u_p: the predictor's output) from the predictor increment u_p - u^n and
the previous step's converged correction, both scaled by the mode's rms of
u_p - u^n.  It is trained online, on the GPU, on the pairs the solver
generates each step (mean squared error, Adam).

``step`` is the reference's time step (src/dnsjax/__main__.py:159-190 with
plane_couette.py:507-582) with one change: the first correction starts
from u_p + guess instead of u_p.  The corrector still iterates to
``corrector_tolerance`` from there, so the guess only moves the starting
point of the same fixed-point iteration.  The guess is applied only while
its measured error on the latest step (before training on that step) is
below ``gate`` times the correction's norm, i.e. while it is closer to the
converged state than the plain predictor.
"""

from __future__ import annotations

from dataclasses import dataclass, field
from math import sqrt

from . import _lib


@dataclass
class LearnedStep:
    corrector_iterations: int
    error: float
    guessed: bool
    guess_rel_error: float | None  # |guess - target| / |target| of this step
    first_correction: float        # norm of the first correction


@dataclass
class LearnedStats:
    steps: list = field(default_factory=list)


class MLP:
    """h = relu(x W1^T + b1), y = h W2^T + b2 over M rows, BF16 weights and
    activations, FP32 accumulation and master weights, Adam; every step of
    the forward and backward pass is a ``dnsb_mlp_*`` kernel.  X (M x
    K1p, BF16) and T (M x N2, FP32) are filled by the caller."""

    def __init__(self, M: int, K1: int, H: int, N2: int, lr: float = 1e-3, seed: int = 0,
                 out_scale: float = 0.1):
        import torch

        self.L = _lib.lib()
        self.M, self.K1, self.H, self.N2 = M, K1, H, N2
        # operand widths padded to multiples of 8 (16-byte rows for the GEMM's
        # vector loads); padded inputs, weights and targets are zero
        self.K1p = (K1 + 7) // 8 * 8
        self.N2p = (N2 + 7) // 8 * 8
        N2p = self.N2p
        self.lr = lr
        g = torch.Generator(device="cpu").manual_seed(seed)
        f32 = dict(dtype=torch.float32, device="cuda")
        bf = dict(dtype=torch.bfloat16, device="cuda")
        W1 = torch.randn(H, self.K1p, generator=g) * sqrt(2.0 / K1)
        W1[:, K1:] = 0.0
        W2 = torch.zeros(N2p, H)
        W2[:N2] = torch.randn(N2, H, generator=g) * (out_scale / sqrt(H))
        self.w = {"W1": W1.to(**f32), "b1": torch.zeros(H, **f32),
                  "W2": W2.to(**f32), "b2": torch.zeros(N2p, **f32)}
        self.wb = {k: self.w[k].to(torch.bfloat16) for k in ("W1", "W2")}
        self.m = {k: torch.zeros_like(v) for k, v in self.w.items()}
        self.v = {k: torch.zeros_like(v) for k, v in self.w.items()}
        self.g = {k: torch.zeros_like(v) for k, v in self.w.items()}
        self.X = torch.zeros(M, self.K1p, **bf)
        self.Hb = torch.empty(M, H, **bf)
        self.dHb = torch.empty(M, H, **bf)
        self.Y = torch.empty(M, N2p, **f32)
        self.T = torch.zeros(M, N2p, **f32)
        self.dYf = torch.empty(M, N2p, **f32)
        self.dYb = torch.empty(M, N2p, **bf)
        self.err = torch.empty(M, **f32)
        self.ref = torch.empty(M, **f32)
        self.adam_step = 0

    @property
    def parameters(self) -> int:
        return self.H * self.K1 + self.H + self.N2 * self.H + self.N2

    def _gemm(self, ta, tb, M, N, K, A, lda, B, ldb, bias=None, relu=0, mask=None, ldm=0,
              Cf=None, Cb=None, ldc=0):
        p = _lib.ptr
        _lib.check(self.L.dnsb_mlp_gemm(
            ta, tb, M, N, K, p(A), lda, p(B), ldb, p(bias) if bias is not None else None, relu,
            p(mask) if mask is not None else None, ldm, p(Cf) if Cf is not None else None,
            p(Cb) if Cb is not None else None, ldc, _lib.stream_handle()))

    def forward(self):
        M = self.M
        self._gemm(0, 0, M, self.H, self.K1p, self.X, self.K1p, self.wb["W1"], self.K1p,
                   bias=self.w["b1"], relu=1, Cb=self.Hb, ldc=self.H)
        self._gemm(0, 0, M, self.N2p, self.H, self.Hb, self.H, self.wb["W2"], self.H,
                   bias=self.w["b2"], Cf=self.Y, ldc=self.N2p)

    def loss(self):
        """Mean-squared-error gradient into dYf / dYb; returns the per-row
        (err, ref) sums of squares."""
        p = _lib.ptr
        _lib.check(self.L.dnsb_mlp_loss_grad(
            p(self.Y), p(self.T), self.M, self.N2p, self.N2p, p(self.dYf), p(self.dYb),
            p(self.err), p(self.ref), _lib.stream_handle()))
        return self.err, self.ref

    def backward(self):
        p = _lib.ptr
        M = self.M
        self._gemm(1, 1, self.N2p, self.H, M, self.dYb, self.N2p, self.Hb, self.H,
                   Cf=self.g["W2"], ldc=self.H)
        _lib.check(self.L.dnsb_mlp_colsum(p(self.dYf), 0, M, self.N2p, self.N2p, p(self.g["b2"]),
                                          _lib.stream_handle()))
        self._gemm(0, 1, M, self.H, self.N2p, self.dYb, self.N2p, self.wb["W2"], self.H,
                   mask=self.Hb, ldm=self.H, Cb=self.dHb, ldc=self.H)
        self._gemm(1, 1, self.H, self.K1p, M, self.dHb, self.H, self.X, self.K1p,
                   Cf=self.g["W1"], ldc=self.K1p)
        _lib.check(self.L.dnsb_mlp_colsum(p(self.dHb), 1, M, self.H, self.H, p(self.g["b1"]),
                                          _lib.stream_handle()))

    def update(self):
        p = _lib.ptr
        self.adam_step += 1
        for k, w in self.w.items():
            wb = self.wb.get(k)
            _lib.check(self.L.dnsb_mlp_adam(
                p(w), p(self.m[k]), p(self.v[k]), p(self.g[k]),
                p(wb) if wb is not None else None, w.numel(), self.lr, 0.9, 0.999, 1e-8,
                self.adam_step, _lib.stream_handle()))

    def train(self, iters: int):
        for it in range(iters):
            if it:
                self.forward()
                self.loss()
            self.backward()
            self.update()


class LearnedGuess:
    """The MLP bound to a plane-Couette flow: features from the spectral
    fields, the guessed prediction, and the learned time step."""

    def __init__(self, flow, hidden: int = 512, lr: float = 1e-3, train_iters: int = 2,
                 gate: float = 0.9, mode_gate: float | None = None, seed: int = 0):
        import torch

        if not hasattr(flow, "imm"):
            raise ValueError("the learned guess is built for plane Couette")
        self.flow = flow
        self.ny = flow.ny
        self.NM = (flow.nz - 1) * (flow.nx // 2)
        self.net = MLP(self.NM, 12 * self.ny + 2, hidden, 6 * self.ny, lr=lr, seed=seed)
        self.train_iters, self.gate, self.mode_gate = train_iters, gate, mode_gate
        self.mode_ok = None  # per mode: 1 where its latest guess error was below mode_gate
        self.kx_max = float(max(abs(flow.fourier.kx_global).max(), 1e-30))
        self.kz_max = float(max(abs(flow.fourier.kz_global).max(), 1e-30))
        self.scale = torch.empty(self.NM, dtype=torch.float32, device="cuda")
        self.last_rel = None  # guess error of the latest step, before training on it

    def features(self, un, up, dprev=None, target=None, s_floor=0.0):
        p = _lib.ptr
        n = self.net
        _lib.check(self.flow._L.dnsb_learned_features(
            self.flow._ctx, p(un), p(up), p(dprev) if dprev is not None else None,
            p(target) if target is not None else None, self.kx_max, self.kz_max,
            float(s_floor), p(n.X), n.K1p, p(n.T), n.N2p, p(self.scale), _lib.stream_handle()))

    def guess(self, up, out):
        p = _lib.ptr
        _lib.check(self.flow._L.dnsb_learned_guess(self.flow._ctx, p(up), p(self.net.Y),
                                                   self.net.N2p, p(self.scale), p(out),
                                                   _lib.stream_handle()))
        return out

    # -- one time step -----------------------------------------------------------
    def step(self, state, dprev, tol, max_iter):
        """One reference time step with the guessed starting point; returns
        (new state, converged correction u^{n+1} - u_p, LearnedStep)."""
        import torch

        f = self.flow
        err = torch.empty(1, dtype=torch.float64, device="cuda")
        r0 = f.get_rhs(state)
        up = f.predict(state, r0)
        inc = torch.linalg.vector_norm(up - state)
        s_floor = 1e-3 * float(inc) / sqrt(up.numel())
        use = self.last_rel is not None and self.last_rel < self.gate
        start = up.clone()
        if use:
            self.features(state, up, dprev, s_floor=s_floor)
            self.net.forward()
            if self.mode_ok is not None:
                self.scale.mul_(self.mode_ok)  # no guess for the other modes
            self.guess(up, start)
        rn = f.get_rhs(start)
        cur = f.correct_fused(state, start, r0, rn, err, out=start)
        e = float(err.item())
        first = e
        c = 0
        while e > tol and c < max_iter:
            rp = rn
            rn = f.get_rhs(cur)
            cur = f.correct_fused(state, cur, rp, rn, err, out=cur)
            c += 1
            e = float(err.item())
        cur, _ = f.correct_velocity(cur)
        delta = cur - up
        # learn from this step's pair; measure the guess first
        self.features(state, up, dprev, target=delta, s_floor=s_floor)
        self.net.forward()
        er, rf = self.net.loss()
        s2 = self.scale.double() ** 2
        rel = float(torch.sqrt((er.double() * s2).sum()
                               / (rf.double() * s2).sum().clamp_min(1e-300)))
        self.last_rel = rel
        if self.mode_gate is not None:
            self.mode_ok = (er < (self.mode_gate ** 2) * rf).float()
        self.net.train(self.train_iters)
        return cur, delta, LearnedStep(c, e, use, rel, first)


def run(flow, state, steps, guess: LearnedGuess, tol=None, max_iter=None):
    """``steps`` learned-guess time steps from ``state``; stops early, like
    the reference loop, when a step does not reach the tolerance."""
    p = flow.params
    tol = p.step.corrector_tolerance if tol is None else tol
    max_iter = p.step.max_corrector_iterations if max_iter is None else max_iter
    stats = LearnedStats()
    dprev = None
    for _ in range(steps):
        state, dprev, st = guess.step(state, dprev, tol, max_iter)
        stats.steps.append(st)
        if not st.error < tol:
            break
    return state, stats
