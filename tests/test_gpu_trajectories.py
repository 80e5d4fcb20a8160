"""Plane-Couette trajectories of the benchmark workloads against the oracle.

The fixtures (``tests/golden/trajectories/*.npz``, made by
``tests/golden/make_trajectories.py``) hold the oracle's run of the
reference's step / corrector loop (``__main__.py:125-203`` with
``plane_couette.py:376-582``) in FP64 from the seeded fields the benchmark
uses, with the influence-matrix operators from the oracle's restatement of
the reference's ``precompute_imm``.  The CUDA path (operators computed on
the GPU) runs the same steps through the host loop and the step graph:

* 64x65x64 (p = 4, Re 400, dt 0.02), 100 steps: the corrector iterations
  of every step identical, E' of every step within 1e-10 relative, the
  low-wavenumber block at steps 10 and 50 and the whole field at step 100
  within 1e-10 relative L2 in every velocity component;
* 128x129x128 (p = 6, Re 1000, dt 0.01), the benchmark's 30-step horizon:
  iterations and E' step for step, the low-wavenumber block at steps 10
  and 30 within 1e-10 in every component;
* the step graph reproduces the host loop's states bit for bit.
"""

import json
from pathlib import Path

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

FIX = Path(__file__).resolve().parent / "golden" / "trajectories"


def _load(name):
    with np.load(FIX / f"{name}.npz") as z:
        d = dict(z)
    return json.loads(str(d.pop("case_json"))), d


def _flow_and_field(c):
    from dnsjax_b200 import initial
    from dnsjax_b200.flows.plane_couette import PlaneCouetteFlow
    from dnsjax_b200.parameters import Parameters

    p = Parameters(phys=dict(system="plane-couette", re=c["re"]),
                   geo=dict(lx=c["lx"], lz=c["lz"]),
                   res=dict(nx=c["nx"], ny=c["ny"], nz=c["nz"], fd_order=c["p"]),
                   step=dict(dt=c["dt"], corrector_tolerance=c["tol"],
                             max_corrector_iterations=c["max_iter"]))
    u0 = initial.couette_field(c["nx"], c["ny"], c["nz"], c["lx"], c["lz"], c["p"],
                               c["seed"], c["kscale"], c["energy"])
    return PlaneCouetteFlow(p), u0


def _block(c, u):
    nkz = c["nz"] - 1
    kzb = c["kz_block"]
    rows = np.concatenate([np.arange(kzb), np.arange(nkz - kzb + 1, nkz)])
    return u[:, rows, :c["kx_block"], :]


def _run_and_compare(name):
    import torch

    from dnsjax_b200 import driver

    c, g = _load(name)
    flow, u0 = _flow_and_field(c)
    steps = c["steps"]
    marks = sorted(set(c["checkpoints"]) | set(c["full"]))
    state = torch.as_tensor(u0, device="cuda")
    iters, energy, done = [], [], 0
    snapshots = {}
    steppers = flow.make_stepper()
    while done < steps:
        state, k, e = driver.step(flow, steppers, state, c["tol"], c["max_iter"])
        assert e <= c["tol"], (done + 1, e)
        done += 1
        iters.append(k)
        energy.append(flow.get_stats(state)["E'"])
        if done in marks:
            snapshots[done] = state.cpu().numpy()
    assert iters == [int(x) for x in g["iterations"]]
    e_rel = np.abs(np.array(energy) - g["energy"]) / g["energy"]
    assert e_rel.max() <= 1e-10, e_rel.max()
    for n in c["checkpoints"]:
        got, want = _block(c, snapshots[n]), g[f"block_{n}"]
        for comp in range(3):
            assert rel_l2(got[comp], want[comp]) <= 1e-10, (n, comp)
    for n in c["full"]:
        for comp in range(3):
            assert rel_l2(snapshots[n][comp], g[f"state_{n}"][comp]) <= 1e-10, (n, comp)
    # the same steps as one step-graph launch each: bitwise the host loop's
    gstate = torch.as_tensor(u0, device="cuda")
    graph = flow.make_step_graph(gstate, tol=c["tol"], max_iter=c["max_iter"])
    g_iters = []
    for _ in range(steps):
        graph.launch()
        g_iters.append(graph.status()[0])
    graph.close()
    assert g_iters == iters
    assert np.array_equal(gstate.cpu().numpy(), snapshots[steps])


def test_couette64_100_steps():
    _run_and_compare("couette64")


def test_couette128_benchmark_horizon():
    _run_and_compare("couette128")
