"""Lockstep ensembles and step graphs: trajectories of different sizes
advanced together (one stream each, one host synchronisation per corrector
round, or one CUDA graph per step with the corrector loop on the device)
give exactly the states and corrector-iteration counts of the same
trajectories stepped one after another by the host-driven loop.  Step graphs
are checked for the triply periodic flows and for plane Couette."""

from math import pi

import pytest

pytestmark = pytest.mark.gpu


def member(n, re, seed):
    from dnsjax_b200 import initial
    from dnsjax_b200.flows.monochromatic import TriplyPeriodicFlow
    from dnsjax_b200.parameters import Parameters

    p = Parameters(phys=dict(system="kolmogorov", re=re),
                   geo=dict(lx=2 * pi, lz=2 * pi), res=dict(nx=n, ny=n, nz=n),
                   step=dict(dt=0.01, corrector_tolerance=1e-10))
    u0 = initial.periodic_field(n, n, n, 2 * pi, 2 * pi, 2 * pi, seed,
                                initial.kolmogorov_spectrum_cfg0, 1e-2)
    return TriplyPeriodicFlow(p, ly=2 * pi), u0


def test_lockstep_equals_sequential():
    import torch

    from dnsjax_b200 import driver
    from dnsjax_b200.ensemble import Ensemble

    spec = [(32, 35.0, 0), (48, 60.0, 1), (32, 75.0, 2), (64, 42.0, 3)]
    built = [member(*s) for s in spec]
    flows = [f for f, _ in built]
    ens = Ensemble(flows, [torch.as_tensor(u, device="cuda") for _, u in built])
    lock_iters = [ens.step().corrector_iterations for _ in range(3)]
    for i, (f, u) in enumerate(built):
        st = f.make_stepper()
        s = torch.as_tensor(u, device="cuda")
        for k in range(3):
            s, c, e = driver.step(f, st, s, f.params.step.corrector_tolerance,
                                  f.params.step.max_corrector_iterations)
            assert c == lock_iters[k][i]
        assert torch.equal(s, ens.states[i]), i


def test_step_graph_equals_driver():
    import torch

    from dnsjax_b200 import driver

    f, u = member(32, 40.0, 5)
    s_eager = torch.as_tensor(u, device="cuda")
    s_graph = torch.as_tensor(u, device="cuda")
    g = f.make_step_graph(s_graph)
    st = f.make_stepper()
    for _ in range(3):
        s_eager, c, e = driver.step(f, st, s_eager, f.params.step.corrector_tolerance,
                                    f.params.step.max_corrector_iterations)
        g.launch()
        it, err = g.status()
        assert it == c and err == e
    assert torch.equal(s_eager, s_graph)
    # a corrector cap below the needed count ends the loop at the cap
    f2, u2 = member(32, 40.0, 5)
    s2 = torch.as_tensor(u2, device="cuda")
    g2 = f2.make_step_graph(s2, max_iter=1)
    g2.launch()
    assert g2.status()[0] == 1
    # a cap of 2 ends the loop in the second iteration of the graph's body;
    # the state matches the host loop with the same cap
    f3, u3 = member(32, 40.0, 5)
    s3 = torch.as_tensor(u3, device="cuda")
    s3_eager = torch.as_tensor(u3, device="cuda")
    g3 = f3.make_step_graph(s3, max_iter=2)
    g3.launch()
    assert g3.status()[0] == 2
    s3_eager, c, _ = driver.step(f3, f3.make_stepper(), s3_eager,
                                 f3.params.step.corrector_tolerance, 2)
    assert c == 2 and torch.equal(s3_eager, s3)


@pytest.mark.parametrize("unroll,max_iter", [(1, 10), (2, 10), (3, 10), (64, 10), (4, 2)])
def test_step_graph_unrolled(unroll, max_iter):
    """Periodic step graphs with corrector iterations held as straight-line
    kernels (fewer, as many and more than the step needs; a cap below the
    unrolled count): the host loop's states and iteration counts."""
    import torch

    from dnsjax_b200 import driver

    f, u = member(48, 60.0, 1)
    s_eager = torch.as_tensor(u, device="cuda")
    s_graph = torch.as_tensor(u, device="cuda")
    g = f.make_step_graph(s_graph, max_iter=max_iter, unroll=unroll)
    st = f.make_stepper()
    for _ in range(3):
        s_eager, c, e = driver.step(f, st, s_eager, f.params.step.corrector_tolerance, max_iter)
        g.launch()
        it, err = g.status()
        assert it == c and err == e
        assert it <= max_iter
    assert torch.equal(s_eager, s_graph)
    g.close()


def test_step_graph_host_round_trip():
    """run_host: the state copied in from pinned host memory and out again
    every step, the copy-out of one step overlapping the copy-in of the
    next, gives the device-resident steps bit for bit."""
    import torch

    f, u = member(32, 40.0, 5)
    s_dev = torch.as_tensor(u, device="cuda")
    g_dev = f.make_step_graph(s_dev)
    f2, _ = member(32, 40.0, 5)
    s_bound = torch.empty_like(s_dev)
    g_host = f2.make_step_graph(s_bound)
    a = torch.empty(s_dev.shape, dtype=s_dev.dtype, pin_memory=True)
    b = torch.empty_like(a, pin_memory=True)
    a.copy_(torch.as_tensor(u))
    for chunks in (8, 3):
        for _ in range(3):
            g_dev.launch()
            g_host.run_host(a, b, chunks=chunks)
            assert g_host.status() == g_dev.status()
            a, b = b, a
    g_host.wait_host()
    torch.cuda.synchronize()
    assert torch.equal(a, s_dev.cpu())


@pytest.mark.parametrize("unroll", [None, 2])
def test_graph_ensemble_equals_sequential(unroll):
    import torch

    from dnsjax_b200 import driver
    from dnsjax_b200.ensemble import Ensemble

    spec = [(32, 35.0, 0), (48, 60.0, 1), (64, 42.0, 3)]
    built = [member(*s) for s in spec]
    ens = Ensemble([f for f, _ in built], [torch.as_tensor(u, device="cuda") for _, u in built],
                   graphs=True, unroll=unroll)
    its = [ens.step().corrector_iterations for _ in range(3)]
    for i, (f, u) in enumerate(built):
        st = f.make_stepper()
        s = torch.as_tensor(u, device="cuda")
        for k in range(3):
            s, c, e = driver.step(f, st, s, f.params.step.corrector_tolerance,
                                  f.params.step.max_corrector_iterations)
            assert c == its[k][i]
        assert torch.equal(s, ens.states[i]), i


def test_graph_ensemble_host_round_trip():
    """step_host (each member's state in from pinned host memory and out
    again on its own stream) gives the device-resident steps bit for bit."""
    import torch

    from dnsjax_b200.ensemble import Ensemble

    spec = [(32, 35.0, 0), (48, 60.0, 1)]
    built = [member(*s) for s in spec]
    dev = Ensemble([f for f, _ in built], [torch.as_tensor(u, device="cuda") for _, u in built],
                   graphs=True)
    built2 = [member(*s) for s in spec]
    hst = Ensemble([f for f, _ in built2],
                   [torch.empty(u.shape, dtype=torch.complex128, device="cuda") for _, u in built2],
                   graphs=True)
    host = [torch.as_tensor(u).pin_memory() for _, u in built2]
    for _ in range(2):
        a = dev.step()
        b = hst.step_host(host, host)
        assert a.corrector_iterations == b.corrector_iterations
    torch.cuda.synchronize()
    for x, h in zip(dev.states, host):
        assert torch.equal(x.cpu(), h)


def couette_member(n, re, seed):
    from dnsjax_b200 import initial
    from dnsjax_b200.flows.plane_couette import PlaneCouetteFlow
    from dnsjax_b200.parameters import Parameters

    p = Parameters(phys=dict(system="plane-couette", re=re),
                   geo=dict(lx=2 * pi, lz=pi), res=dict(nx=n, ny=n + 1, nz=n, fd_order=4),
                   step=dict(dt=0.02, corrector_tolerance=1e-10))
    u0 = initial.couette_field(n, n + 1, n, 2 * pi, pi, 4, seed, 8.0, 1e-3)
    return PlaneCouetteFlow(p), u0


def test_couette_step_graph_equals_driver():
    import torch

    from dnsjax_b200 import driver

    f, u = couette_member(64, 400.0, 2)
    s_eager = torch.as_tensor(u, device="cuda")
    s_graph = torch.as_tensor(u, device="cuda")
    g = f.make_step_graph(s_graph)
    st = f.make_stepper()
    for _ in range(3):
        s_eager, c, e = driver.step(f, st, s_eager, f.params.step.corrector_tolerance,
                                    f.params.step.max_corrector_iterations)
        g.launch()
        it, err = g.status()
        assert it == c and err == e
    f.check_status()
    assert torch.equal(s_eager, s_graph)
    g.close()
    g2 = f.make_step_graph(torch.as_tensor(u, device="cuda"), max_iter=0)
    g2.launch()
    assert g2.status()[0] == 0


@pytest.mark.parametrize("unroll,max_iter", [(1, 60), (2, 60), (5, 60), (64, 60), (5, 2)])
def test_couette_step_graph_unrolled(unroll, max_iter):
    """Corrector iterations held as straight-line kernels ahead of the WHILE
    node (fewer, as many as, and more than the step needs; odd and even
    counts; a cap below the unrolled count): the host loop's states bit for
    bit and its iteration counts."""
    import torch

    from dnsjax_b200 import driver

    f, u = couette_member(64, 400.0, 2)
    s_eager = torch.as_tensor(u, device="cuda")
    s_graph = torch.as_tensor(u, device="cuda")
    g = f.make_step_graph(s_graph, max_iter=max_iter, unroll=unroll)
    st = f.make_stepper()
    its = []
    for _ in range(3):
        s_eager, c, e = driver.step(f, st, s_eager, f.params.step.corrector_tolerance, max_iter)
        g.launch()
        it, err = g.status()
        assert it == c and err == e
        its.append(it)
    f.check_status()
    assert torch.equal(s_eager, s_graph)
    if max_iter == 2:
        assert its == [2, 2, 2]
    g.close()


def test_couette_graph_ensemble_equals_sequential():
    import torch

    from dnsjax_b200 import driver
    from dnsjax_b200.ensemble import Ensemble

    spec = [(32, 300.0, 1), (48, 500.0, 3), (32, 200.0, 4)]
    built = [couette_member(*s) for s in spec]
    ens = Ensemble([f for f, _ in built], [torch.as_tensor(u, device="cuda") for _, u in built],
                   graphs=True)
    its = [ens.step().corrector_iterations for _ in range(2)]
    for i, (f, u) in enumerate(built):
        st = f.make_stepper()
        s = torch.as_tensor(u, device="cuda")
        for k in range(2):
            s, c, e = driver.step(f, st, s, f.params.step.corrector_tolerance,
                                  f.params.step.max_corrector_iterations)
            assert c == its[k][i]
        assert torch.equal(s, ens.states[i]), i


def test_worklist_ensemble_equals_step_graphs():
    """The work-list ensemble (one launch per stage for all members, the
    corrector loop on the device while any member iterates) against each
    member's own step graph: the same states bit for bit and the same
    iteration counts, over 4 steps of members of three sizes and different
    Re, including a member with a corrector cap it reaches (max_iter 1)."""
    import torch

    from dnsjax_b200 import _lib

    spec = [(32, 35.0, 0), (48, 60.0, 1), (64, 42.0, 3), (32, 75.0, 2), (48, 30.0, 4)]
    built = [member(*s) for s in spec]
    flows = [f for f, _ in built]
    caps = [10, 10, 10, 1, 10]
    states = [torch.as_tensor(u, device="cuda") for _, u in built]

    L = _lib.lib()
    n = len(flows)
    ctxs = (_lib.C.c_void_p * n)(*[f._ctx.value for f in flows])
    sts = (_lib.C.c_void_p * n)(*[f._check(x) for f, x in zip(flows, states)])
    tols = (_lib.C.c_double * n)(*[1e-10] * n)
    mis = (_lib.C.c_int * n)(*caps)
    h = _lib.C.c_void_p()
    _lib.check(L.dnsb_ensemble_create(ctxs, sts, n, tols, mis, 1, _lib.C.byref(h)))
    its_w = []
    for _ in range(4):
        _lib.check(L.dnsb_ensemble_step(h, _lib.stream_handle()))
        its = (_lib.C.c_int * n)()
        errs = (_lib.C.c_double * n)()
        _lib.check(L.dnsb_ensemble_status(h, its, errs, _lib.stream_handle()))
        its_w.append(list(its))
    L.dnsb_ensemble_destroy(h)
    assert any(k[3] == 1 for k in its_w)  # the capped member stopped at its cap
    for i, (f, u) in enumerate(built):
        s = torch.as_tensor(u, device="cuda")
        g = f.make_step_graph(s, tol=1e-10, max_iter=caps[i])
        for k in range(4):
            g.launch()
            assert g.status()[0] == its_w[k][i], (i, k)
        g.close()
        assert torch.equal(s, states[i]), i


def test_worklist_ensemble_class():
    """Ensemble(worklist=True) steps the same states as Ensemble(graphs=True)."""
    import torch

    from dnsjax_b200.ensemble import Ensemble

    spec = [(32, 35.0, 7), (64, 50.0, 8), (48, 45.0, 9)]
    built = [member(*s) for s in spec]
    flows = [f for f, _ in built]
    a = Ensemble(flows, [torch.as_tensor(u, device="cuda") for _, u in built], worklist=True)
    b = Ensemble(flows, [torch.as_tensor(u, device="cuda") for _, u in built], graphs=True)
    for _ in range(3):
        sa, sb = a.step(), b.step()
        assert sa.corrector_iterations == sb.corrector_iterations
    for x, y in zip(a.states, b.states):
        assert torch.equal(x, y)
    a.close()
