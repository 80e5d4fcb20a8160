"""Slab decomposition host logic over two processes (gloo, CPU).

The kernels need a GPU; here each rank's flow is a stand-in that records the
calls the slab driver makes, so the multi-process logic is checked on the
host: every rank learns every other rank's receive buffers, the RHS phases
run in order with a barrier between consecutive phases (the same collectives
in the same order on every rank), the corrector error is the square root of
the norm shares summed over the ranks, so every rank takes the same
corrector decisions (src/dnsjax/__main__.py:166-180), and the shards
tile kx.
"""

import os

import torch.multiprocessing as mp


class FakeFlow:
    """One rank's flow: buffers are integers, the RHS phases are recorded,
    the squared-norm share of rank r after n corrector calls is
    (r + 1) * 4**-n (so the summed error falls by 2 per iteration)."""

    device = "cpu"

    def __init__(self, slab):
        import types

        self.nranks, self.rank = slab
        self.params = types.SimpleNamespace(step=types.SimpleNamespace(
            corrector_tolerance=1e-3, max_corrector_iterations=60))
        nkx = 8 // self.nranks
        self.kx_range = (self.rank * nkx, (self.rank + 1) * nkx)
        self.kx_axis = 1
        self.calls = []
        self.ncorr = 0

    def _new(self):
        import torch

        return torch.zeros(3, self.kx_range[1] - self.kx_range[0])

    def slab_buffers(self):
        return 1000 + self.rank, 2000 + self.rank

    def slab_connect(self, bx, bk):
        self.connected = (list(bx), list(bk))

    def rhs_phase(self, state, out, phase):
        self.calls.append(("phase", phase))
        return out

    def predict(self, state, rhs):
        return state.clone()

    def correct_fused(self, sp, p, rp, rn, share, out=None):
        share.fill_((self.rank + 1) * 4.0 ** (-self.ncorr))
        self.ncorr += 1
        return p

    def correct_velocity(self, s):
        return s, None


def _worker(rank, world, port, out):
    import torch
    import torch.distributed as dist

    from dnsjax_b200 import driver
    from dnsjax_b200.slab import Slab, TorchComm

    class TestComm(TorchComm):
        """TorchComm whose buffer handles are the integers themselves."""

        def __init__(self, log):
            super().__init__(device="cpu")
            self.log = log

        def barrier(self):
            self.log.append(("barrier",))
            super().barrier()

        @staticmethod
        def export(ptr):
            return int(ptr).to_bytes(64, "little")

        @staticmethod
        def open(handle):
            return int.from_bytes(handle, "little") + 10**6

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        log = []
        comm = TestComm(log)
        slab = Slab(FakeFlow, world, comm=comm)
        f = slab.flows[0]
        f.calls = log  # one timeline for phases and barriers
        whole = torch.arange(3 * 8, dtype=torch.float64).reshape(3, 8)
        (mine,) = slab.scatter(whole)
        slab.get_rhs([mine])
        rhs_timeline = list(log)
        del log[:]
        st = slab.make_stepper()
        _, c, e = driver.step(slab, st, [mine], 1e-3, 60)
        out[rank] = dict(connected=f.connected, opened=list(slab._opened),
                         rhs=rhs_timeline, iters=c, err=e, shard=mine.tolist(),
                         barriers=sum(1 for x in log if x[0] == "barrier"))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_slab_two_ranks_host_logic():
    import math
    import socket

    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    r0, r1 = out[0], out[1]
    # every rank addresses every rank's buffers: its own directly, the
    # other's through the opened handle
    assert r0["connected"] == ([1000, 10**6 + 1001], [2000, 10**6 + 2001])
    assert r1["connected"] == ([10**6 + 1000, 1001], [10**6 + 2000, 2001])
    assert r0["opened"] == [10**6 + 1001, 10**6 + 2001]
    # phases 0, 1, 2 with a barrier between consecutive phases
    want = [("phase", 0), ("barrier",), ("phase", 1), ("barrier",), ("phase", 2)]
    assert r0["rhs"] == r1["rhs"] == want
    # the error after the predictor and n corrector iterations is
    # sqrt(1 + 2) 2**-n; both ranks stop at the same n (11: the first with
    # sqrt(3) 2**-n <= 1e-3)
    n = next(k for k in range(60) if math.sqrt(3.0) * 2.0 ** -k <= 1e-3)
    assert n == 11
    assert r0["iters"] == r1["iters"] == n
    assert abs(r0["err"] - math.sqrt(3.0) * 2.0 ** -n) < 1e-15
    assert r0["err"] == r1["err"]
    # two barriers per RHS, two RHS per predictor step plus one per iteration
    assert r0["barriers"] == r1["barriers"] == 2 * (2 + r0["iters"])
    # the shards tile kx
    assert r0["shard"] == [[0, 1, 2, 3], [8, 9, 10, 11], [16, 17, 18, 19]]
    assert r1["shard"] == [[4, 5, 6, 7], [12, 13, 14, 15], [20, 21, 22, 23]]
