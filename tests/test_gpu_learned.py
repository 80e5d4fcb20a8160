"""The learned corrector guess (plane Couette): its BF16 MLP kernels against
the CPU oracle (oracle/mlp.py) and FP64 products, its training, and what it
gains over the method without it.

* The GEMM: the tcgen05 kernel (K-contiguous operands; ragged tiles, split
  K, the full-size first layer) and the mma.sync kernels of the transposed
  layouts, with their epilogues, against FP64 products of the same BF16
  values; split-K results identical run to run.
* Forward pass, loss and every gradient of two- and three-layer networks
  against the oracle with the same BF16 rounding points (relative L2 below
  1e-2: the GPU accumulates in FP32, which can move a BF16 rounding by one
  unit), one Adam update, and bitwise-identical gradients on a repeat.
* Training on a synthetic linear target lowers the loss tenfold.
* Plane Couette 32x33x32: pretrained on steps of other seeded fields, the
  guessed start converges every step to the tolerance, stays within 1e-8 of
  the plain trajectory, and the corrector iterations with and without the
  guess are recorded.
* The graph form of the learned step (LearnedStepGraph: the corrector loop
  and the FP32 -> FP64 switch on the device) gives the host-driven step's
  states bit for bit, with the same iteration counts, RHS precisions,
  first errors and gating decisions: mixed with the gate, mixed with the
  guess applied every step, FP64 without the network, an iteration cap, and
  a tolerance below the FP32 floor (the stall test moves every step to
  FP64), and the first correction without the restart (N(u^n) in the
  previous-RHS slot), with and without corrector iterations held as
  straight-line kernels.
"""

import json
from math import pi

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def bf16_tensor(a):
    import torch

    return torch.as_tensor(np.asarray(a, np.float32), device="cuda").to(torch.bfloat16)


def as64(t):
    return t.float().cpu().numpy().astype(np.float64)


def _gemm(L, ta, tb, M, N, K, A, lda, B, ldb, Cf, ldc, bias=None, relu=0, mask=None, ldm=0,
          Cb=None, work=None, status=None):
    from dnsjax_b200 import _lib

    p = _lib.ptr
    _lib.check(L.dnsb_mlp_gemm(ta, tb, M, N, K, p(A), lda, p(B), ldb,
                               p(bias) if bias is not None else None, relu,
                               p(mask) if mask is not None else None, ldm,
                               p(Cf) if Cf is not None else None,
                               p(Cb) if Cb is not None else None, ldc,
                               p(work) if work is not None else None,
                               work.numel() if work is not None else 0,
                               p(status) if status is not None else None, _lib.stream_handle()))


# (70, 45, 100): unaligned leading dimensions, the 64 x 64 kernel; (200,
# 136, 264): ragged 128 x 128 tiles (tcgen05 when neither operand is
# transposed); (64, 96, 4096): split K on tcgen05.
@pytest.mark.parametrize("M,N,K", [(70, 45, 100), (200, 136, 264), (64, 96, 4096)])
@pytest.mark.parametrize("ta,tb", [(0, 0), (1, 1), (0, 1)])
def test_mlp_gemm_layouts(ta, tb, M, N, K):
    import torch

    from dnsjax_b200 import _lib

    L = _lib.lib()
    rng = np.random.default_rng(ta * 2 + tb)
    Am = rng.standard_normal((M, K))
    Bn = rng.standard_normal((N, K))
    A = bf16_tensor(Am.T if ta else Am).contiguous()
    B = bf16_tensor(Bn.T if tb else Bn).contiguous()
    lda, ldb = (M if ta else K), (N if tb else K)
    ref = (as64(A).T if ta else as64(A)) @ (as64(B) if tb else as64(B).T)
    Cf = torch.empty(M, N, dtype=torch.float32, device="cuda")
    work = torch.empty(8 * M * N, dtype=torch.float32, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    _gemm(L, ta, tb, M, N, K, A, lda, B, ldb, Cf, N, work=work, status=status)
    got = Cf.double().cpu().numpy()
    assert np.abs(got - ref).max() <= 1e-5 * np.abs(ref).max()
    again = torch.empty_like(Cf)
    _gemm(L, ta, tb, M, N, K, A, lda, B, ldb, again, N, work=work, status=status)
    assert torch.equal(again, Cf)  # fixed-order reductions
    # epilogue: bias, relu, mask, BF16 copy
    bias = torch.as_tensor(rng.standard_normal(N), dtype=torch.float32, device="cuda")
    mask = bf16_tensor(rng.standard_normal((M, N)))
    Cb = torch.empty(M, N, dtype=torch.bfloat16, device="cuda")
    _gemm(L, ta, tb, M, N, K, A, lda, B, ldb, Cf, N, bias=bias, relu=1, mask=mask, ldm=N, Cb=Cb,
          work=work, status=status)
    want = np.maximum(ref + bias.double().cpu().numpy(), 0.0) * (as64(mask) > 0)
    got = Cf.double().cpu().numpy()
    assert np.abs(got - want).max() <= 1e-5 * np.abs(want).max()
    assert torch.equal(Cb, Cf.to(torch.bfloat16))
    assert int(status.item()) == 0


def test_tc_gemm_full_size_layer():
    """The first layer at 128x129x128: 8128 modes x 1552 inputs -> 640, on
    tcgen05, against an FP64 product of the same BF16 values."""
    import torch

    from dnsjax_b200 import _lib

    L = _lib.lib()
    M, N, K = 8128, 640, 1552
    g = torch.Generator(device="cpu").manual_seed(7)
    A = torch.randn(M, K, generator=g).to(torch.bfloat16).cuda()
    B = (torch.randn(N, K, generator=g) / 30).to(torch.bfloat16).cuda()
    bias = torch.randn(N, generator=g).float().cuda()
    Cf = torch.empty(M, N, dtype=torch.float32, device="cuda")
    Cb = torch.empty(M, N, dtype=torch.bfloat16, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    _gemm(L, 0, 0, M, N, K, A, K, B, K, Cf, N, bias=bias, relu=1, Cb=Cb, status=status)
    ref = torch.relu(A.double() @ B.double().t() + bias.double())
    err = (Cf.double() - ref).abs().max().item()
    assert err <= 1e-5 * ref.abs().max().item(), err
    assert torch.equal(Cb, Cf.to(torch.bfloat16))
    assert int(status.item()) == 0


@pytest.mark.parametrize("M,sizes", [(150, [70, 48, 30]), (256, [72, 64, 48, 40])])
def test_mlp_gradients_match_oracle(M, sizes):
    """M = 150: unaligned rows (the mma.sync kernels in the backward pass);
    M = 256 with three layers: every product on tcgen05."""
    import torch

    from dnsjax_b200.learned import MLP
    from oracle import mlp as om

    rng = np.random.default_rng(5)
    net = MLP(M, sizes, lr=1e-3, seed=3, out_scale=1.0)
    nl = len(sizes) - 1
    X = rng.standard_normal((M, net.K1p))
    X[:, net.K1:] = 0.0
    net.X.copy_(bf16_tensor(X))
    T = rng.standard_normal((M, net.N2))
    net.T[:, :net.N2] = torch.as_tensor(T, dtype=torch.float32)
    net.forward()
    err, _ = net.loss()
    net.backward()
    Ws = [net.w[f"W{l + 1}"].double().cpu().numpy() for l in range(nl)]
    bs = [net.w[f"b{l + 1}"].double().cpu().numpy() for l in range(nl)]
    loss, gW, gb = om.loss_and_grads_layers(as64(net.X), Ws, bs, net.T.double().cpu().numpy())
    assert abs(float(err.double().sum()) / M - loss) <= 1e-4 * loss
    if net.N2p > net.N2:  # padded output rows get no gradient
        assert float(net.g[f"W{nl}"][net.N2:].abs().max()) == 0.0
    for l in range(nl):
        for k, ref in ((f"W{l + 1}", gW[l]), (f"b{l + 1}", gb[l])):
            got = net.g[k].double().cpu().numpy()
            rel = np.linalg.norm(got - ref) / np.linalg.norm(ref)
            assert rel < 1e-2, (k, rel)
    # the same gradients bit for bit on a repeat (fixed-order reductions)
    first = {k: v.clone() for k, v in net.g.items()}
    net.forward()
    net.loss()
    net.backward()
    for k in first:
        assert torch.equal(first[k], net.g[k]), k
    # one Adam update against the oracle's
    w0 = {k: v.double().cpu().numpy() for k, v in net.w.items()}
    gg = {k: v.double().cpu().numpy() for k, v in net.g.items()}
    net.update()
    for k in net.w:
        want, _, _ = om.adam(w0[k], 0.0, 0.0, gg[k], 1, 1e-3)
        got = net.w[k].double().cpu().numpy()
        assert np.abs(got - want).max() <= 1e-6 * max(1.0, np.abs(want).max()), k
    for k in net.wb:
        assert torch.equal(net.wb[k], net.w[k].to(torch.bfloat16))
        assert torch.equal(net.wt[k], net.wb[k].t())
    assert net.pipeline_status() == 0


def test_mlp_training_lowers_loss():
    import torch

    from dnsjax_b200.learned import MLP

    rng = np.random.default_rng(9)
    net = MLP(1024, [64, 128, 32], lr=3e-3, seed=1)
    X = rng.standard_normal((1024, net.K1p)) * (np.arange(net.K1p) < 64)
    A = rng.standard_normal((net.K1p, 32)) / 8.0
    net.X.copy_(bf16_tensor(X))
    net.T.copy_(torch.as_tensor(as64(net.X) @ A, dtype=torch.float32))
    net.forward()
    l0 = float(net.loss()[0].sum())
    net.train(1)
    for _ in range(299):
        net.forward()
        net.loss()
        net.train(1)
    net.forward()
    l1 = float(net.loss()[0].sum())
    assert l1 < 0.1 * l0, (l0, l1)


def test_learned_couette_run(tmp_path):
    import torch

    from dnsjax_b200 import driver, initial, learned
    from dnsjax_b200.flows.plane_couette import PlaneCouetteFlow
    from dnsjax_b200.parameters import Parameters

    p = Parameters(phys=dict(system="plane-couette", re=400.0),
                   geo=dict(lx=2 * pi, lz=pi), res=dict(nx=32, ny=33, nz=32, fd_order=4),
                   step=dict(dt=0.02, corrector_tolerance=1e-10, max_corrector_iterations=60))
    flow = PlaneCouetteFlow(p)
    lg = learned.LearnedGuess(flow, hidden=(128, 128), seed=0)
    for seed in (11, 12, 13):  # training fields: other seeds than the run's
        u = initial.couette_field(32, 33, 32, 2 * pi, pi, 4, seed, 8.0, 1e-3)
        lg.collect(torch.as_tensor(u, device="cuda"), 8, 1e-10, 60)
    losses = lg.pretrain(30)
    assert losses[-1] < 0.5 * losses[0], losses
    u0 = initial.couette_field(32, 33, 32, 2 * pi, pi, 4, 1, 8.0, 1e-3)
    n = 16
    u_l, stats = learned.run(flow, torch.as_tensor(u0, device="cuda"), n, lg)
    lg.enabled = False  # the same restarted step from the predictor, no network
    u_0, stats0 = learned.run(flow, torch.as_tensor(u0, device="cuda"), n, lg)
    r = driver.run(flow, torch.as_tensor(u0, device="cuda"), n)
    assert len(stats.steps) == n and all(s.error <= 1e-10 for s in stats.steps)
    assert all(s.error <= 1e-10 for s in stats0.steps)
    assert r.converged and r.steps == n
    for u in (u_l, u_0):
        d = torch.linalg.vector_norm(u - r.state) / torch.linalg.vector_norm(r.state)
        assert float(d) < 1e-8
    record = dict(plain_iterations=r.corrector_iterations,
                  restart_iterations=[s.corrector_iterations for s in stats0.steps],
                  learned_iterations=[s.corrector_iterations for s in stats.steps],
                  guessed=[s.guessed for s in stats.steps],
                  guess_rel_error=[s.guess_rel_error for s in stats.steps],
                  pretrain_losses=[losses[0], losses[-1]], parameters=lg.net.parameters)
    (tmp_path / "learned_gain.json").write_text(json.dumps(record))
    print(json.dumps(record))


@pytest.mark.parametrize("form,unroll", [("mixed-gated", 0), ("mixed-guess", 0),
                                         ("fp64-no-network", 0), ("mixed-cap", 0),
                                         ("mixed-stall", 0), ("mixed-norestart", 0),
                                         ("mixed-norestart", 3), ("mixed-gated", 3),
                                         ("fp64-no-network", 2), ("mixed-cap", 5),
                                         ("mixed-guess", 64), ("mixed-stall", 6)])
def test_learned_step_graph_equals_host_step(form, unroll):
    import torch

    from dnsjax_b200 import initial, learned
    from dnsjax_b200.flows.plane_couette import PlaneCouetteFlow
    from dnsjax_b200.parameters import Parameters

    p = Parameters(phys=dict(system="plane-couette", re=400.0),
                   geo=dict(lx=2 * pi, lz=pi), res=dict(nx=32, ny=33, nz=32, fd_order=4),
                   step=dict(dt=0.02, corrector_tolerance=1e-10, max_corrector_iterations=60))
    flow = PlaneCouetteFlow(p)
    mixed = form.startswith("mixed")
    # mixed-stall: the switch at a tolerance below the FP32 rounding floor,
    # so only the stall test (no contraction over two corrections) moves the
    # iteration to FP64
    stall_only = form == "mixed-stall"
    lg = learned.LearnedGuess(flow, hidden=(64, 64), seed=0,
                              switch=(1e-11 if stall_only else 1e-5) if mixed else None,
                              gate=None if form == "mixed-guess" else 0.9,
                              restart=form != "mixed-norestart")
    u = initial.couette_field(32, 33, 32, 2 * pi, pi, 4, 11, 8.0, 1e-3)
    lg.collect(torch.as_tensor(u, device="cuda"), 6, 1e-10, 60)
    lg.pretrain(5)
    lg.enabled = form != "fp64-no-network"
    tol = (1e-11 if stall_only else 1e-8) if mixed else 1e-10
    mi = 2 if form == "mixed-cap" else 60
    u0 = initial.couette_field(32, 33, 32, 2 * pi, pi, 4, 1, 8.0, 1e-3)
    n = 12

    lg.last_rel, lg._since = None, 0
    s, dprev, host = torch.as_tensor(u0, device="cuda"), None, []
    for _ in range(n):
        s, dprev, st = lg.step(s, dprev, tol, mi)
        host.append(st)

    lg.last_rel, lg._since = None, 0
    g_state = torch.as_tensor(u0, device="cuda")
    g = lg.make_step_graph(g_state, tol, mi, unroll=unroll)
    dev = [g.step() for _ in range(n)]
    g.close()
    for k, (a, b) in enumerate(zip(host, dev)):
        assert a.corrector_iterations == b.corrector_iterations, k
        assert a.error == b.error and a.first_correction == b.first_correction, k
        assert (a.rhs_fp32, a.rhs_fp64) == (b.rhs_fp32, b.rhs_fp64), k
        assert a.guessed == b.guessed and a.guess_rel_error == b.guess_rel_error, k
    assert torch.equal(s, g_state)
    if form == "mixed-cap":
        assert all(x.corrector_iterations <= 2 for x in dev)
    if mixed:
        assert all(x.rhs_fp32 >= 2 for x in dev)
    else:
        assert all(x.rhs_fp32 == 0 for x in dev)
    if form == "mixed-gated":
        assert dev[0].guessed and dev[0].guess_rel_error is not None
    if form == "mixed-guess":
        assert all(x.guessed for x in dev)
    if stall_only:
        assert all(x.rhs_fp64 > 0 for x in dev)  # every step finished in FP64
