"""The learned corrector guess (plane Couette): its BF16 MLP kernels against
the CPU oracle (oracle/mlp.py), its training, and what it gains over the
plain method.

* The tensor-core GEMM in the three operand layouts the network uses, with
  its epilogues, against FP64 products of the same BF16 values.
* Forward pass, loss and every gradient of the MLP against the oracle with
  the same BF16 rounding points (relative L2 below 1e-2: the GPU
  accumulates in FP32, which can move a BF16 rounding by one unit), and one
  Adam update.
* Training on a synthetic linear target lowers the loss tenfold.
* Plane Couette 32x33x32 with the learned guess: every step converges to
  the tolerance, the trajectory stays within 1e-8 of the plain one, the
  guess's error falls as it trains, and the corrector iterations with and
  without it are recorded (the gain the network brings).
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


# (70, 45, 100): unaligned leading dimensions, the 64 x 64 kernel; (200,
# 136, 264): the 128 x 128 kernel with ragged tiles; (64, 96, 4096): its
# split-K path.
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
    p = _lib.ptr
    _lib.check(L.dnsb_mlp_gemm(ta, tb, M, N, K, p(A), lda, p(B), ldb, None, 0, None, 0, p(Cf),
                               None, N, _lib.stream_handle()))
    got = Cf.double().cpu().numpy()
    assert np.abs(got - ref).max() <= 1e-5 * np.abs(ref).max()
    # epilogue: bias, relu, mask, BF16 copy
    bias = torch.as_tensor(rng.standard_normal(N), dtype=torch.float32, device="cuda")
    mask = bf16_tensor(rng.standard_normal((M, N)))
    Cb = torch.empty(M, N, dtype=torch.bfloat16, device="cuda")
    _lib.check(L.dnsb_mlp_gemm(ta, tb, M, N, K, p(A), lda, p(B), ldb, p(bias), 1, p(mask), N,
                               p(Cf), p(Cb), N, _lib.stream_handle()))
    want = np.maximum(ref + bias.double().cpu().numpy(), 0.0) * (as64(mask) > 0)
    got = Cf.double().cpu().numpy()
    assert np.abs(got - want).max() <= 1e-5 * np.abs(want).max()
    assert torch.equal(Cb, Cf.to(torch.bfloat16))


def test_mlp_gradients_match_oracle():
    import torch

    from dnsjax_b200.learned import MLP
    from oracle import mlp as om

    rng = np.random.default_rng(5)
    net = MLP(M=150, K1=70, H=48, N2=30, lr=1e-3, seed=3, out_scale=1.0)
    X = rng.standard_normal((150, net.K1p))
    X[:, net.K1:] = 0.0
    net.X.copy_(bf16_tensor(X))
    T = rng.standard_normal((150, 30))
    net.T[:, :30] = torch.as_tensor(T, dtype=torch.float32)
    net.forward()
    err, _ = net.loss()
    net.backward()
    w = {k: v.double().cpu().numpy() for k, v in net.w.items()}
    loss, g = om.loss_and_grads(as64(net.X), w["W1"], w["b1"], w["W2"], w["b2"],
                                net.T.double().cpu().numpy())
    assert abs(float(err.double().sum()) / 150 - loss) <= 1e-4 * loss
    assert net.N2p == 32 and float(net.g["W2"][30:].abs().max()) == 0.0
    for k in ("W1", "b1", "W2", "b2"):
        got = net.g[k].double().cpu().numpy()
        rel = np.linalg.norm(got - g[k]) / np.linalg.norm(g[k])
        assert rel < 1e-2, (k, rel)
    # one Adam update against the oracle's
    w0 = {k: v.double().cpu().numpy() for k, v in net.w.items()}
    gg = {k: v.double().cpu().numpy() for k, v in net.g.items()}
    net.update()
    for k in net.w:
        want, _, _ = om.adam(w0[k], 0.0, 0.0, gg[k], 1, 1e-3)
        got = net.w[k].double().cpu().numpy()
        assert np.abs(got - want).max() <= 1e-6 * max(1.0, np.abs(want).max()), k
    assert torch.equal(net.wb["W1"], net.w["W1"].to(torch.bfloat16))


def test_mlp_training_lowers_loss():
    import torch

    from dnsjax_b200.learned import MLP

    rng = np.random.default_rng(9)
    net = MLP(M=1024, K1=64, H=128, N2=32, lr=3e-3, seed=1)
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
    u0 = initial.couette_field(32, 33, 32, 2 * pi, pi, 4, 1, 8.0, 1e-3)
    flow = PlaneCouetteFlow(p)
    lg = learned.LearnedGuess(flow, hidden=128, train_iters=4, seed=0)
    n = 16
    u_l, stats = learned.run(flow, torch.as_tensor(u0, device="cuda"), n, lg)
    r = driver.run(flow, torch.as_tensor(u0, device="cuda"), n)
    assert len(stats.steps) == n and all(s.error <= 1e-10 for s in stats.steps)
    assert r.converged and r.steps == n
    d = torch.linalg.vector_norm(u_l - r.state) / torch.linalg.vector_norm(r.state)
    assert float(d) < 1e-8
    rels = [s.guess_rel_error for s in stats.steps]
    assert min(rels[n // 2:]) < rels[0]
    record = dict(plain_iterations=r.corrector_iterations,
                  learned_iterations=[s.corrector_iterations for s in stats.steps],
                  guessed=[s.guessed for s in stats.steps], guess_rel_error=rels,
                  parameters=lg.net.parameters)
    (tmp_path / "learned_gain.json").write_text(json.dumps(record))
    print(json.dumps(record))
