"""Learned corrector guess for plane Couette.

A per-(kz, kx)-mode MLP with two hidden layers (12 Ny + 2 -> 640 -> 640 ->
6 Ny; 1.9M parameters at 128x129x128), BF16 weights and activations and
FP32 accumulation on the tcgen05 tensor cores (``dnsb_mlp_*``,
``csrc/mlp_tc.cu``, ``csrc/learned.cu``).  For every mode it guesses the
converged corrector correction u^{n+1} - u_p (u_p: the predictor's output)
from the predictor increment u_p - u^n and the previous step's converged
correction, both scaled by the mode's rms of u_p - u^n.

Training: ``LearnedGuess.collect`` runs the plain FP64 solver (the
reference's loop) from seeded initial fields and keeps every step's
per-mode (predictor, previous correction, converged correction) triples on
the GPU; ``pretrain`` fits the network to them (mean squared error, Adam),
all with this package's own forward and backward kernels.  ``step`` can
also keep training online on each step's pair.

``step`` is the reference's time step (src/dnsjax/__main__.py:159-190 with
plane_couette.py:507-582) started from the guessed state u_p + guess: the
corrector iterations of ``iterate_correction`` (timestep.py:96-120) run
from there to ``corrector_tolerance``, so the guess only moves the starting
point of the same fixed-point iteration and the converged state is the
same to within the tolerance.  With ``restart`` (the default) the guessed
state is treated as the previous iterate, so its own RHS fills both RHS
slots of the first correction (the reference's predict_and_correct keeps
N(u^n) in the first slot).  With ``switch`` set (the mixed form), the RHS
runs in FP32 until the correction norm falls below ``switch`` or the FP32
iteration stops contracting, and in FP64 from then on within the step; with
the switch at the tolerance, the FP32 RHS carries the whole iteration unless
it stagnates above the tolerance.

``LearnedStepGraph`` (``LearnedGuess.make_step_graph``) is the same step with
the corrector on the device: the predictor and the corrector loop are CUDA
graphs, the precision switch is decided by a control kernel after every
correction, and the host synchronises once per step.
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
    rhs_fp32: int = 0              # RHS evaluations of the step in FP32
    rhs_fp64: int = 0              # and in FP64


@dataclass
class LearnedStats:
    steps: list = field(default_factory=list)


def _pad8(n: int) -> int:
    return (n + 7) // 8 * 8


class MLP:
    """y = W_L relu(... relu(W_1 x + b_1) ...) + b_L over M rows, BF16
    weights and activations, FP32 accumulation and master weights, Adam;
    every step of the forward and backward pass is a ``dnsb_mlp_*`` kernel.
    ``sizes`` = [inputs, hidden..., outputs].  X (M x K1p, BF16) and T (M x
    N2p, FP32) are filled by the caller; widths are padded to multiples of
    8 (16-byte rows), the padding of inputs, weights and targets is zero.

    Every product is C = A B^T with both operands K-contiguous (the tcgen05
    kernel); the backward pass feeds it transposed copies of the
    activations and gradients (``dnsb_mlp_transpose``) and keeps a
    transposed BF16 copy of every weight matrix.  Reductions (split-K
    partials, bias gradients) run in a fixed order, so training is
    reproducible run to run."""

    def __init__(self, M: int, sizes, lr: float = 1e-3, seed: int = 0, out_scale: float = 0.1):
        import torch

        self.L = _lib.lib()
        sizes = [int(s) for s in sizes]
        if len(sizes) < 2:
            raise ValueError("sizes = [inputs, hidden..., outputs]")
        self.M, self.sizes = M, sizes
        self.dims = [_pad8(s) for s in sizes]
        self.K1, self.N2 = sizes[0], sizes[-1]
        self.K1p, self.N2p = self.dims[0], self.dims[-1]
        self.H = sizes[1] if len(sizes) > 2 else None
        self.nl = len(sizes) - 1
        self.lr = lr
        g = torch.Generator(device="cpu").manual_seed(seed)
        f32 = dict(dtype=torch.float32, device="cuda")
        bf = dict(dtype=torch.bfloat16, device="cuda")
        self.w = {}
        for l in range(self.nl):
            din, dout = sizes[l], sizes[l + 1]
            W = torch.zeros(self.dims[l + 1], self.dims[l])
            if l < self.nl - 1:
                W[:dout, :din] = torch.randn(dout, din, generator=g) * sqrt(2.0 / din)
            else:
                W[:dout, :din] = torch.randn(dout, din, generator=g) * (out_scale / sqrt(din))
            self.w[f"W{l + 1}"] = W.to(**f32)
            self.w[f"b{l + 1}"] = torch.zeros(self.dims[l + 1], **f32)
        self.wb = {f"W{l + 1}": self.w[f"W{l + 1}"].to(torch.bfloat16) for l in range(self.nl)}
        self.wt = {k: v.t().contiguous() for k, v in self.wb.items()}
        self.m = {k: torch.zeros_like(v) for k, v in self.w.items()}
        self.v = {k: torch.zeros_like(v) for k, v in self.w.items()}
        self.g = {k: torch.zeros_like(v) for k, v in self.w.items()}
        # activations: acts[0] = X (input), acts[l] = hidden layer l output
        self.acts = [torch.zeros(M, self.dims[0], **bf)]
        for l in range(1, self.nl):
            self.acts.append(torch.empty(M, self.dims[l], **bf))
        self.X = self.acts[0]
        self.dacts = [None] + [torch.empty(M, self.dims[l], **bf) for l in range(1, self.nl)]
        self.Y = torch.empty(M, self.N2p, **f32)
        self.T = torch.zeros(M, self.N2p, **f32)
        self.dYf = torch.empty(M, self.N2p, **f32)
        self.dYb = torch.empty(M, self.N2p, **bf)
        self.err = torch.empty(M, **f32)
        self.ref = torch.empty(M, **f32)
        dmax = max(self.dims)
        self.tA = torch.empty(dmax * M, **bf)  # transposed gradient
        self.tB = torch.empty(dmax * M, **bf)  # transposed activation
        wmax = max(self.dims[l] * self.dims[l + 1] for l in range(self.nl))
        self.work = torch.empty(max(4 * wmax, 128 * dmax), **f32)
        self.status = torch.zeros(1, dtype=torch.int32, device="cuda")
        self.adam_step = 0

    @property
    def parameters(self) -> int:
        return sum(self.sizes[l] * self.sizes[l + 1] + self.sizes[l + 1] for l in range(self.nl))

    @property
    def layers(self) -> list:
        return list(self.sizes)

    def _gemm(self, M, N, K, A, lda, B, ldb, bias=None, relu=0, mask=None, ldm=0, Cf=None,
              Cb=None, ldc=0, split=False):
        """C[M][N] = sum_k A[m][k] B[n][k] (both K-contiguous)."""
        p = _lib.ptr
        work, nwork = (p(self.work), self.work.numel()) if split else (None, 0)
        _lib.check(self.L.dnsb_mlp_gemm(
            0, 0, M, N, K, p(A), lda, p(B), ldb, p(bias) if bias is not None else None, relu,
            p(mask) if mask is not None else None, ldm, p(Cf) if Cf is not None else None,
            p(Cb) if Cb is not None else None, ldc, work, nwork, p(self.status),
            _lib.stream_handle()))

    def _transpose(self, A, R, C, out):
        _lib.check(self.L.dnsb_mlp_transpose(_lib.ptr(A), R, C, C, _lib.ptr(out), R,
                                             _lib.stream_handle()))

    def _colsum(self, A, bf16, N, out):
        p = _lib.ptr
        _lib.check(self.L.dnsb_mlp_colsum(p(A), int(bf16), self.M, N, N, p(out), p(self.work),
                                          self.work.numel(), _lib.stream_handle()))

    def forward(self):
        M, d = self.M, self.dims
        for l in range(self.nl):
            W, b = self.wb[f"W{l + 1}"], self.w[f"b{l + 1}"]
            if l < self.nl - 1:
                self._gemm(M, d[l + 1], d[l], self.acts[l], d[l], W, d[l], bias=b, relu=1,
                           Cb=self.acts[l + 1], ldc=d[l + 1])
            else:
                self._gemm(M, d[l + 1], d[l], self.acts[l], d[l], W, d[l], bias=b, Cf=self.Y,
                           ldc=d[l + 1])

    def capture_forward(self):
        """Capture ``forward`` (its GEMM launches, bound to this network's
        buffers) as a CUDA graph; ``replay_forward`` then runs it with one
        launch.  Re-capture is not needed after training: the graph reads the
        weight buffers, which Adam updates in place."""
        import torch

        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            self.forward()  # first launches (kernel attributes) outside the capture
        torch.cuda.current_stream().wait_stream(side)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.forward()
        self._fwd_graph = g

    def replay_forward(self):
        g = getattr(self, "_fwd_graph", None)
        if g is None:
            self.forward()
        else:
            g.replay()

    def loss(self):
        """Mean-squared-error gradient into dYf / dYb; returns the per-row
        (err, ref) sums of squares."""
        p = _lib.ptr
        _lib.check(self.L.dnsb_mlp_loss_grad(
            p(self.Y), p(self.T), self.M, self.N2p, self.N2p, p(self.dYf), p(self.dYb),
            p(self.err), p(self.ref), _lib.stream_handle()))
        return self.err, self.ref

    def backward(self):
        M, d = self.M, self.dims
        cur = self.dYb
        for l in range(self.nl - 1, -1, -1):
            dout, din = d[l + 1], d[l]
            # weight gradient g[o][i] = sum_m cur[m][o] acts[l][m][i]
            self._transpose(cur, M, dout, self.tA)
            self._transpose(self.acts[l], M, din, self.tB)
            self._gemm(dout, din, M, self.tA, M, self.tB, M, Cf=self.g[f"W{l + 1}"], ldc=din,
                       split=True)
            if l == self.nl - 1:
                self._colsum(self.dYf, False, dout, self.g[f"b{l + 1}"])
            else:
                self._colsum(cur, True, dout, self.g[f"b{l + 1}"])
            if l > 0:
                # input gradient (cur W) masked by the relu of layer l
                self._gemm(M, din, dout, cur, dout, self.wt[f"W{l + 1}"], dout,
                           mask=self.acts[l], ldm=din, Cb=self.dacts[l], ldc=din)
                cur = self.dacts[l]

    def update(self):
        p = _lib.ptr
        self.adam_step += 1
        for k, w in self.w.items():
            wb = self.wb.get(k)
            _lib.check(self.L.dnsb_mlp_adam(
                p(w), p(self.m[k]), p(self.v[k]), p(self.g[k]),
                p(wb) if wb is not None else None, w.numel(), self.lr, 0.9, 0.999, 1e-8,
                self.adam_step, _lib.stream_handle()))
            if wb is not None:
                R, C = wb.shape
                self._transpose(wb, R, C, self.wt[k])

    def train(self, iters: int):
        """``iters`` Adam iterations on the current X, T (the first reuses
        the forward pass and loss the caller ran)."""
        for it in range(iters):
            if it:
                self.forward()
                self.loss()
            self.backward()
            self.update()

    def pipeline_status(self) -> int:
        """Bit 0: a tensor-core pipeline wait gave up (synchronises)."""
        return int(self.status.item())


class LearnedGuess:
    """The MLP bound to a plane-Couette flow: features from the spectral
    fields, the guessed prediction, data collection, pretraining and the
    learned time step."""

    def __init__(self, flow, hidden=(640, 640), lr: float = 1e-3, seed: int = 0,
                 restart: bool = True, switch: float | None = None, gate: float | None = 0.9,
                 train_iters: int = 0):
        import torch

        if not hasattr(flow, "imm"):
            raise ValueError("the learned guess is built for plane Couette")
        if isinstance(hidden, int):
            hidden = (hidden,)
        self.flow = flow
        self.ny = flow.ny
        self.NM = (flow.nz - 1) * (flow.nx // 2)
        self.net = MLP(self.NM, [12 * self.ny + 2, *hidden, 6 * self.ny], lr=lr, seed=seed)
        self.restart, self.switch, self.gate = restart, switch, gate
        # FP32 iterations stop when e > stall * the error two corrections
        # back: the corrector's errors fall in pairs (from the seeded
        # 128x129x128 field, FP64 or FP32 alike: 3.3e-4, 6.4e-6, 6.4e-6,
        # 4.7e-7, 2.4e-7), so a pause of one iteration is not the FP32 floor
        self.stall = 0.8
        self.recheck = 8      # while gated off, measure the guess every recheck steps
        self.trace = None     # list: (iteration, error, fp32) of every correction
        self._since = 0
        self.train_iters = train_iters
        self.kx_max = float(max(abs(flow.fourier.kx_global).max(), 1e-30))
        self.kz_max = float(max(abs(flow.fourier.kz_global).max(), 1e-30))
        self.scale = torch.empty(self.NM, dtype=torch.float32, device="cuda")
        self.last_rel = None  # guess error of the latest step, measured after it
        self.enabled = True   # False: the same step with no guess (u_p as start)
        self.data = []        # (X, T, scale) of collected steps

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

    def _s_floor(self, up, state):
        import torch

        inc = torch.linalg.vector_norm(up - state)
        return 1e-3 * float(inc) / sqrt(up.numel())

    def measure(self, state, up, dprev, delta, s_floor) -> float:
        """Relative error of the network's guess of ``delta`` (= converged
        state - u_p) on this step; leaves the step's features and target in
        the network's X, T."""
        import torch

        self.features(state, up, dprev, target=delta, s_floor=s_floor)
        self.net.replay_forward()
        er, rf = self.net.loss()
        s2 = self.scale.double() ** 2
        return float(torch.sqrt((er.double() * s2).sum()
                                / (rf.double() * s2).sum().clamp_min(1e-300)))

    # -- data and pretraining --------------------------------------------------
    def collect(self, state, steps: int, tol: float, max_iter: int):
        """Run ``steps`` plain FP64 reference steps from ``state`` and keep each
        step's training triple (features of u^n, u_p, previous correction;
        target u^{n+1} - u_p) on the GPU.  Returns the final state."""
        import torch

        f = self.flow
        err = torch.empty(1, dtype=torch.float64, device="cuda")
        was32 = f.rhs_fp32
        f.set_rhs_precision(False)
        dprev = None
        try:
            for _ in range(steps):
                r0 = f.get_rhs(state)
                up = f.predict(state, r0)
                rn = f.get_rhs(up)
                cur = f.correct_fused(state, up.clone(), r0, rn, err)
                c, e = 0, float(err.item())
                while e > tol and c < max_iter:
                    rp, rn = rn, f.get_rhs(cur)
                    cur = f.correct_fused(state, cur, rp, rn, err, out=cur)
                    c, e = c + 1, float(err.item())
                if not e <= tol:
                    break
                cur, _ = f.correct_velocity(cur)
                delta = cur - up
                self.features(state, up, dprev, target=delta, s_floor=self._s_floor(up, state))
                self.data.append((self.net.X.clone(), self.net.T.clone(), self.scale.clone()))
                dprev, state = delta, cur
        finally:
            f.set_rhs_precision(was32)
        return state

    def pretrain(self, epochs: int) -> list:
        """``epochs`` passes over the collected steps, one Adam iteration per
        step; returns the mean loss of each epoch (synchronises once per
        epoch)."""
        import torch

        n = self.net
        losses = []
        for _ in range(epochs):
            tot = torch.zeros((), dtype=torch.float64, device="cuda")
            for X, T, _s in self.data:
                n.X.copy_(X)
                n.T.copy_(T)
                n.forward()
                er, _ = n.loss()
                tot += er.double().sum()
                n.backward()
                n.update()
            losses.append(float(tot) / max(1, len(self.data) * n.M))
        n.capture_forward()
        return losses

    # -- one time step -----------------------------------------------------------
    def make_step_graph(self, state, tol: float, max_iter: int,
                        unroll: int | None = None) -> "LearnedStepGraph":
        """The graph form of ``step`` bound to ``state`` (see
        LearnedStepGraph); ``switch``, ``stall`` and ``restart`` are fixed
        when it is made; ``unroll`` corrector iterations are held as
        straight-line kernels (PlaneCouetteFlow.set_graph_unroll)."""
        return self.flow._with_unroll(
            unroll, lambda: LearnedStepGraph(self, state, tol, max_iter))

    def _plan(self):
        """(use the guess, measure it, steps since the last measurement) for
        the next step: the guess is used while its latest measured error is
        below the gate; while gated off it is re-measured every ``recheck``
        steps; with online training every step is measured.  Depends only on
        earlier steps, so a caller can know it before the step runs."""
        use = self.enabled and (self.gate is None or self.last_rel is None
                                or self.last_rel < self.gate)
        gated_off = self.gate is not None and not use and self.last_rel is not None
        since = self._since + 1 if gated_off else 0
        measure = self.enabled and (self.train_iters > 0 or (
            self.gate is not None and (not gated_off or since >= self.recheck)))
        if gated_off and measure:
            since = 0
        return use, measure, since

    def step(self, state, dprev, tol, max_iter, measure: bool | None = None):
        """One time step started from the guessed state; returns (new state,
        converged correction u^{n+1} - u_p, LearnedStep)."""
        import torch

        f = self.flow
        err = torch.empty(1, dtype=torch.float64, device="cuda")
        mixed = self.switch is not None
        n32 = n64 = 0

        def rhs(u):
            nonlocal n32, n64
            if f.rhs_fp32:
                n32 += 1
            else:
                n64 += 1
            return f.get_rhs(u)

        use, planned, since = self._plan()
        if measure is None:
            measure, self._since = planned, since
        f.set_rhs_precision(mixed)
        r0 = rhs(state)
        up = f.predict(state, r0)
        s_floor = self._s_floor(up, state)
        start = up.clone()
        if use:
            self.features(state, up, dprev, s_floor=s_floor)
            self.net.replay_forward()
            self.guess(up, start)
        rn = rhs(start)
        cur = f.correct_fused(state, start, rn if self.restart else r0, rn, err, out=start)
        e = float(err.item())
        first = e
        c = 0
        e_prev = e_prev2 = float("inf")
        while e > tol and c < max_iter:
            # one way to FP64 for the rest of the step: once below the switch,
            # or when the FP32 iteration stops contracting over two
            # corrections (its rounding floor)
            if mixed and f.rhs_fp32 and (e <= self.switch or e > self.stall * e_prev2):
                f.set_rhs_precision(False)
            rp, rn = rn, rhs(cur)
            cur = f.correct_fused(state, cur, rp, rn, err, out=cur)
            c += 1
            e_prev2, e_prev, e = e_prev, e, float(err.item())
            if self.trace is not None:
                self.trace.append((c, e, int(f.rhs_fp32)))
        f.set_rhs_precision(False)
        cur, _ = f.correct_velocity(cur)
        delta = cur - up
        rel = None
        if measure:
            rel = self.measure(state, up, dprev, delta, s_floor)
            self.last_rel = rel
            if self.train_iters:
                self.net.train(self.train_iters)
        return cur, delta, LearnedStep(c, e, use, rel, first, n32, n64)


class LearnedStepGraph:
    """``LearnedGuess.step`` with the corrector on the device: two CUDA
    graphs per step (``dnsb_couette_mixed_graph_create``) bound to
    ``state``, which every ``step()`` advances in place.

    The first graph runs the RHS of u^n and the predictor; when the guess is
    used, the features, the network's forward pass and the guessed start
    are launched between the two graphs on the same stream; the second graph
    runs the restarted first correction, the corrector loop (FP32 RHS until
    the switch, then FP64, chosen on the device after every correction) and
    copies the converged state into ``state``.  A step synchronises the host
    once (the status), plus once more on steps that use or measure the guess
    (the scale floor of the features).  The states, iteration counts and
    gating decisions are those of ``LearnedGuess.step`` bit for bit.
    ``reset()`` forgets the previous step's correction (as ``dprev=None``)."""

    def __init__(self, guess: LearnedGuess, state, tol: float, max_iter: int):
        import torch

        f = guess.flow
        self.lg, self.flow, self.state = guess, f, state
        self.up, self.cur = f._new(), f._new()
        self._d = (torch.empty_like(state), torch.empty_like(state))
        self._un = None
        self._dprev = None
        self._k = 0
        mixed = guess.switch is not None
        h = _lib.C.c_void_p()
        _lib.check(f._L.dnsb_couette_mixed_graph_create(
            f._ctx, f._check(state), f._check(self.up), f._check(self.cur), float(tol),
            int(max_iter), 1 if mixed else 0, float(guess.switch) if mixed else 0.0,
            float(guess.stall), 1 if guess.restart else 0, _lib.C.byref(h)))
        self._h = h

    def reset(self) -> None:
        self._dprev = None

    def snapshot(self):
        """Copies of the bound state and the previous step's correction."""
        return (self.state.clone(), None if self._dprev is None else self._dprev.clone())

    def restore(self, snap) -> None:
        state, dprev = snap
        self.state.copy_(state)
        if dprev is None:
            self._dprev = None
        else:
            self._dprev = self._d[self._k]
            self._dprev.copy_(dprev)

    def step(self, measure: bool | None = None) -> LearnedStep:
        import torch

        lg, f, L = self.lg, self.flow, self.flow._L
        stream = _lib.stream_handle()
        use, planned, since = lg._plan()
        if measure is None:
            measure, lg._since = planned, since
        _lib.check(L.dnsb_mixed_graph_predict(self._h, stream))
        s_floor = lg._s_floor(self.up, self.state) if (use or measure) else 0.0
        if measure:
            if self._un is None:
                self._un = torch.empty_like(self.state)
            self._un.copy_(self.state)
        if use:
            lg.features(self.state, self.up, self._dprev, s_floor=s_floor)
            lg.net.replay_forward()
            lg.guess(self.up, self.cur)
        _lib.check(L.dnsb_mixed_graph_correct(self._h, stream))
        it, err, first = _lib.C.c_int(), _lib.C.c_double(), _lib.C.c_double()
        n32, n64 = _lib.C.c_int(), _lib.C.c_int()
        _lib.check(L.dnsb_mixed_graph_status(self._h, _lib.C.byref(it), _lib.C.byref(err),
                                             _lib.C.byref(first), _lib.C.byref(n32),
                                             _lib.C.byref(n64), stream))
        rel = None
        delta = None
        if measure:
            delta = self._delta()
            rel = lg.measure(self._un, self.up, self._dprev, delta, s_floor)
            lg.last_rel = rel
            if lg.train_iters:
                lg.net.train(lg.train_iters)
        nuse, nmeasure, _ = lg._plan()
        if nuse or nmeasure:
            self._dprev = delta if delta is not None else self._delta()
        else:
            self._dprev = None
        return LearnedStep(it.value, err.value, use, rel, first.value, n32.value, n64.value)

    def _delta(self):
        """u^{n+1} - u_p of the step just run, in the buffer the previous
        step's correction does not occupy."""
        import torch

        self._k ^= 1
        out = self._d[self._k]
        torch.sub(self.state, self.up, out=out)
        return out

    def close(self) -> None:
        if getattr(self, "_h", None):
            self.flow._L.dnsb_mixed_graph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


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


def forward_rate(M: int = 8128, sizes=(1550, 640, 640, 774), reps: int = 20) -> dict:
    """Inference rate of the network's GEMMs at the 128x129x128 sizes: three
    forward passes, then CUDA-graph replays of the forward timed with CUDA
    events (``python -c "from dnsjax_b200.learned import forward_rate;
    print(forward_rate())"``)."""
    import torch

    net = MLP(M, list(sizes))
    net.X.normal_()
    for _ in range(3):
        net.forward()
    torch.cuda.synchronize()
    net.capture_forward()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        net.replay_forward()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    flops = 2.0 * M * sum(sizes[i] * sizes[i + 1] for i in range(len(sizes) - 1))
    return {"ms": ms, "tflops": flops / (ms * 1e-3) / 1e12, "flops": flops,
            "status": net.pipeline_status()}
