"""Slab decomposition (dnsjax_b200.slab) with every rank emulated on one GPU.

The slab RHS -- z inverse storing into every rank's padded-z share, x pass
storing into every rank's kx share, the column passes on the local kx modes
-- is the single-GPU RHS bit for bit: every column and row transform is the
same arithmetic, only where it is stored differs.  Whole time steps (the
reference loop, src/dnsjax/__main__.py:125-203, with the norm summed over
the ranks) match the single-GPU steps to rounding with the same corrector
iterations.  Sizes follow the reference's slab constraints
(src/dnsjax/sharding.py:107-129): nx/2 and the padded nz divisible by the
number of ranks.
"""

from math import pi

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def dev(a):
    import torch

    return torch.as_tensor(np.ascontiguousarray(a), device="cuda")


def couette_params(nx, ny, nz, p_ord, re, dt, tol=1e-10, max_iter=60):
    from dnsjax_b200.parameters import Parameters

    return Parameters(phys=dict(system="plane-couette", re=re), geo=dict(lx=2 * pi, lz=pi),
                      res=dict(nx=nx, ny=ny, nz=nz, fd_order=p_ord),
                      step=dict(dt=dt, corrector_tolerance=tol, max_corrector_iterations=max_iter))


def periodic_params(n, re, dt, tol=1e-10, max_iter=10):
    from dnsjax_b200.parameters import Parameters

    return Parameters(phys=dict(system="kolmogorov", re=re), geo=dict(lx=2 * pi, lz=2 * pi),
                      res=dict(nx=n, ny=n, nz=n),
                      step=dict(dt=dt, corrector_tolerance=tol, max_corrector_iterations=max_iter))


def couette_case(nx, ny, nz, p_ord, re, dt, energy, kscale, seed):
    from dnsjax_b200 import initial

    p = couette_params(nx, ny, nz, p_ord, re, dt)
    u0 = initial.couette_field(nx, ny, nz, 2 * pi, pi, p_ord, seed, kscale, energy)
    return p, u0


def periodic_case(n, re, dt, energy, seed):
    from dnsjax_b200 import initial

    p = periodic_params(n, re, dt)
    u0 = initial.periodic_field(n, n, n, 2 * pi, 2 * pi, 2 * pi, seed,
                                initial.kolmogorov_spectrum_cfg0, energy)
    return p, u0


@pytest.mark.parametrize("nranks", [1, 2, 4, 8])
def test_couette_slab_rhs_bitwise_32(nranks):
    from dnsjax_b200.flows.plane_couette import PlaneCouetteFlow
    from dnsjax_b200.slab import Slab

    p, u0 = couette_case(32, 33, 32, 4, 400.0, 0.02, 1e-3, 8.0, 3)
    whole = PlaneCouetteFlow(p)
    u = dev(u0)
    ref = whole.get_rhs(u)
    slab = Slab(lambda **k: PlaneCouetteFlow(p, **k), nranks)
    got = slab.gather(slab.get_rhs(slab.scatter(u)))
    assert got.shape == ref.shape
    assert bool((got == ref).all())


@pytest.mark.parametrize("nranks", [2, 4, 8])
def test_couette_slab_rhs_bitwise_128(nranks):
    from dnsjax_b200.flows.plane_couette import PlaneCouetteFlow
    from dnsjax_b200.slab import Slab

    p, u0 = couette_case(128, 129, 128, 6, 1000.0, 0.01, 5e-2, 32.0, 4)
    whole = PlaneCouetteFlow(p)
    u = dev(u0)
    ref = whole.get_rhs(u)
    slab = Slab(lambda **k: PlaneCouetteFlow(p, **k), nranks)
    got = slab.gather(slab.get_rhs(slab.scatter(u)))
    assert bool((got == ref).all())


@pytest.mark.parametrize("nranks", [1, 2, 4, 8])
def test_periodic_slab_rhs_bitwise_32(nranks):
    from dnsjax_b200.flows.monochromatic import TriplyPeriodicFlow
    from dnsjax_b200.slab import Slab

    p, u0 = periodic_case(32, 40.0, 0.01, 1e-2, 0)
    whole = TriplyPeriodicFlow(p)
    u = dev(u0)
    ref = whole.get_rhs(u)
    slab = Slab(lambda **k: TriplyPeriodicFlow(p, **k), nranks)
    got = slab.gather(slab.get_rhs(slab.scatter(u)))
    assert bool((got == ref).all())


def test_periodic_slab_rhs_bitwise_128():
    from dnsjax_b200.flows.monochromatic import TriplyPeriodicFlow
    from dnsjax_b200.slab import Slab

    p, u0 = periodic_case(128, 100.0, 0.005, 0.5, 2)
    whole = TriplyPeriodicFlow(p)
    u = dev(u0)
    ref = whole.get_rhs(u)
    slab = Slab(lambda **k: TriplyPeriodicFlow(p, **k), 4)
    got = slab.gather(slab.get_rhs(slab.scatter(u)))
    assert bool((got == ref).all())


def _compare_runs(whole, slab, u0, steps):
    import torch

    from dnsjax_b200 import driver

    tol = whole.params.step.corrector_tolerance
    mi = whole.params.step.max_corrector_iterations
    st_w, st_s = whole.make_stepper(), slab.make_stepper()
    uw = dev(u0)
    us = slab.scatter(uw.clone())
    for _ in range(steps):
        uw, cw, ew = driver.step(whole, st_w, uw, tol, mi)
        us, cs, es = driver.step(slab, st_s, us, tol, mi)
        assert cs == cw
        assert abs(es - ew) <= 1e-12 * max(ew, 1e-300) + 1e-14
    got = slab.gather(us)
    for c in range(3):
        d = torch.linalg.vector_norm(got[c] - uw[c]).item()
        n = torch.linalg.vector_norm(uw[c]).item()
        assert d <= 1e-12 * n, (c, d / n)


def test_couette_slab_steps_64():
    """Plane Couette 64x65x64 (p = 4, Re 400, dt 0.02): 10 steps of the
    reference loop on 4 slab ranks against the single-GPU steps."""
    from dnsjax_b200.flows.plane_couette import PlaneCouetteFlow
    from dnsjax_b200.slab import Slab

    p, u0 = couette_case(64, 65, 64, 4, 400.0, 0.02, 1e-3, 8.0, 1)
    whole = PlaneCouetteFlow(p)
    slab = Slab(lambda **k: PlaneCouetteFlow(p, **k), 4)
    _compare_runs(whole, slab, u0, 10)


def test_periodic_slab_steps_32():
    """Kolmogorov 32^3 (Re 40, dt 0.01): 10 steps on 2 slab ranks against
    the single-GPU steps; the mean mode and the kx = 0 norm weight live on
    rank 0 only."""
    from dnsjax_b200.flows.monochromatic import TriplyPeriodicFlow
    from dnsjax_b200.slab import Slab

    p, u0 = periodic_case(32, 40.0, 0.01, 1e-2, 0)
    whole = TriplyPeriodicFlow(p)
    slab = Slab(lambda **k: TriplyPeriodicFlow(p, **k), 2)
    _compare_runs(whole, slab, u0, 10)


def test_slab_stats_match_whole():
    """get_stats over the ranks: each rank's sums added over the ranks give
    the whole flow's E' (Couette) and E, I, D, E' (Kolmogorov, whose forced
    modes live on the rank holding kx = 0)."""
    from dnsjax_b200.flows.monochromatic import TriplyPeriodicFlow
    from dnsjax_b200.flows.plane_couette import PlaneCouetteFlow
    from dnsjax_b200.slab import Slab

    p, u0 = couette_case(32, 33, 32, 4, 400.0, 0.02, 1e-3, 8.0, 3)
    whole = PlaneCouetteFlow(p)
    slab = Slab(lambda **k: PlaneCouetteFlow(p, **k), 4)
    u = dev(u0)
    e_w = whole.get_stats(u)["E'"]
    e_s = slab.get_stats(slab.scatter(u))["E'"]
    assert abs(e_s - e_w) <= 1e-13 * e_w
    p, u0 = periodic_case(32, 40.0, 0.01, 1e-2, 0)
    whole = TriplyPeriodicFlow(p)
    slab = Slab(lambda **k: TriplyPeriodicFlow(p, **k), 2)
    u = dev(u0)
    sw = whole.get_stats(u)
    ss = slab.get_stats(slab.scatter(u))
    for k in ("E", "I", "D", "E'"):
        assert abs(ss[k] - sw[k]) <= 1e-12 * abs(sw[k]) + 1e-15, k


def test_slab_refusals():
    from dnsjax_b200 import _lib
    from dnsjax_b200.flows.plane_couette import PlaneCouetteFlow

    p, u0 = couette_case(32, 33, 32, 4, 400.0, 0.02, 1e-3, 8.0, 3)
    f = PlaneCouetteFlow(p, slab=(2, 1))
    u = dev(np.ascontiguousarray(u0[:, :, 8:16]))
    # not connected yet
    with pytest.raises(_lib.DnsbError, match="not connected"):
        f.rhs_phase(u, f._new(), 0)
    # the whole-context entry points refuse a slab context
    with pytest.raises(_lib.DnsbError, match="phases"):
        f.get_rhs(u)
    with pytest.raises(_lib.DnsbError, match="host loop"):
        f.make_step_graph(u)
    with pytest.raises(_lib.DnsbError, match="FP64"):
        f.set_rhs_precision(True)
    # nz_p = 48 is not a multiple of 5 ranks; nx/2 = 16 is not either
    with pytest.raises(_lib.DnsbError, match="multiples of nranks"):
        PlaneCouetteFlow(p, slab=(5, 0))


def _bench(args, env_extra=None):
    import json
    import os
    import subprocess
    import sys
    from pathlib import Path

    root = Path(__file__).resolve().parents[1]
    env = dict(os.environ)
    env.update(env_extra or {})
    r = subprocess.run([sys.executable, str(root / "bench.py"), *args], cwd=root, env=env,
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_bench_slab_emulated():
    """bench.py --parallel slab with 4 ranks emulated on this GPU."""
    out = _bench(["--parallel", "slab", "--slab-emulate", "4", "--workload", "couette64",
                  "--steps", "3", "--warmup", "1"])
    assert out["value"] > 0 and out["scaling"] == "strong"
    assert "emulated" in out["config"]["parallelism"]
    assert out["diagnostics"]["last_error"] <= 1e-10


def test_bench_slab_one_process_nccl():
    """bench.py --parallel slab as one torch.distributed rank (NCCL barriers,
    the CUDA IPC export of the receive buffers)."""
    import socket

    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    out = _bench(["--parallel", "slab", "--workload", "couette64", "--steps", "3",
                  "--warmup", "1"],
                 {"RANK": "0", "WORLD_SIZE": "1", "LOCAL_RANK": "0",
                  "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    assert out["value"] > 0 and out["n_gpus"] == 1
    assert out["config"]["parallelism"] == "slab over 1 GPUs"
