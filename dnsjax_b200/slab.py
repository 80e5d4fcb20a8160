"""One trajectory over several GPUs: the reference's slab decomposition.

The reference shards every spectral array on kx and the physical (padded)
grid on z, with a reshard between the column transforms and the x transform
in each direction (src/dnsjax/sharding.py:107-129, src/dnsjax/fft.py:193-392;
jax ``shard_map`` + ``reshard``); the corrector's norm is a sum over all
shards.  Here each rank is a slab context (``slab=(nranks, rank)`` on the flow
classes) whose z-inverse and x-pass kernels store their outputs straight into
the receive buffer of the rank that owns them -- the reshard is fused into
those kernels -- so the RHS is three phases with a cross-rank barrier
between them; the norm shares are summed over the ranks and square-rooted.

``Slab`` holds the ranks of this process and exposes the flow interface the
driver uses (``make_stepper``, ``correct_velocity``, ``get_rhs``,
``predict``, ``correct_fused``, ``norm``) over *sharded states*: a list with
one tensor per rank held here.  Two communicators:

* ``LocalComm`` -- every rank in this process, on one device; the barrier is
  the order of the one stream, the shares are summed in a loop.  This is how
  the decomposition runs (and is tested) on a single GPU.
* ``TorchComm`` -- one rank per process under ``torch.distributed`` (NCCL),
  each on its own GPU: the receive buffers are exchanged as CUDA IPC handles
  and mapped with peer access, the barrier is an NCCL all-reduce of one
  element on the current stream (stream-ordered: every rank's kernels before
  it have completed when it completes), and the norm shares are all-reduced.
"""

from __future__ import annotations

from . import _lib


class LocalComm:
    """All ranks in this process (one device)."""

    nprocs = 1

    def barrier(self) -> None:  # stream order is the barrier
        return None

    def sum_(self, t) -> None:  # the local sum is already the total
        return None

    def exchange_buffers(self, bufs):
        """Every rank's (bx, bk) receive buffers from those of the ranks held
        here: all of them, addressed directly."""
        return [b[0] for b in bufs], [b[1] for b in bufs], []


class TorchComm:
    """One rank per process over torch.distributed (NCCL, one GPU each)."""

    def __init__(self, device: str = "cuda"):
        import torch
        import torch.distributed as dist

        self.dist = dist
        self.rank = dist.get_rank()
        self.nprocs = dist.get_world_size()
        self._tick = torch.zeros(1, dtype=torch.float64, device=device)

    def barrier(self) -> None:
        self.dist.all_reduce(self._tick)

    def sum_(self, t) -> None:
        self.dist.all_reduce(t)

    def all_gather_bytes(self, b: bytes) -> list:
        out = [None] * self.nprocs
        self.dist.all_gather_object(out, b)
        return out

    def exchange_buffers(self, bufs):
        """Every rank's (bx, bk) receive buffers: this process's own, the
        others' mapped from their CUDA IPC handles (returned third, to be
        unmapped on close)."""
        (bx0, bk0), = bufs
        allh = self.all_gather_bytes(self.export(bx0) + self.export(bk0))
        bx, bk, opened = [], [], []
        for r, h in enumerate(allh):
            if r == self.rank:
                bx.append(bx0)
                bk.append(bk0)
            else:
                px, pk = self.open(h[:64]), self.open(h[64:])
                opened += [px, pk]
                bx.append(px)
                bk.append(pk)
        return bx, bk, opened

    @staticmethod
    def export(ptr: int) -> bytes:
        return ipc_handle(ptr)

    @staticmethod
    def open(handle: bytes) -> int:
        return ipc_open(handle)


def ipc_handle(ptr: int) -> bytes:
    h = (_lib.C.c_char * 64)()
    _lib.check(_lib.lib().dnsb_ipc_handle(_lib.C.c_void_p(ptr), h))
    return bytes(h)


def ipc_open(handle: bytes) -> int:
    p = _lib.C.c_void_p()
    buf = (_lib.C.c_char * 64).from_buffer_copy(handle)
    _lib.check(_lib.lib().dnsb_ipc_open(buf, _lib.C.byref(p)))
    return p.value


class Slab:
    """``nranks`` slab ranks of one flow; ``make_flow(slab=(nranks, r))``
    builds rank r (e.g. ``lambda **k: PlaneCouetteFlow(params, **k)``).
    Without ``comm`` every rank lives in this process; with a ``TorchComm``
    this process holds rank ``comm.rank`` of ``comm.nprocs``."""

    def __init__(self, make_flow, nranks: int, comm=None):
        self.nranks = int(nranks)
        self.comm = LocalComm() if comm is None else comm
        if comm is None:
            self.ranks = list(range(self.nranks))
        else:
            if comm.nprocs != self.nranks:
                raise ValueError("one slab rank per process: nranks must equal the world size")
            self.ranks = [comm.rank]
        self.flows = [make_flow(slab=(self.nranks, r)) for r in self.ranks]
        self.params = self.flows[0].params
        self.device = getattr(self.flows[0], "device", "cuda")
        self._opened = []
        self._connect()

    def _connect(self) -> None:
        bx, bk, self._opened = self.comm.exchange_buffers([f.slab_buffers() for f in self.flows])
        for f in self.flows:
            f.slab_connect(bx, bk)

    def close(self) -> None:
        for p in self._opened:
            _lib.check(_lib.lib().dnsb_ipc_close(_lib.C.c_void_p(p)))
        self._opened = []

    # -- sharding of whole-problem tensors ---------------------------------------
    def kx_axis(self) -> int:
        return self.flows[0].kx_axis

    def scatter(self, state):
        """The shards of a whole-problem spectral tensor held by this process."""
        ax = self.kx_axis()
        out = []
        for f in self.flows:
            k0, k1 = f.kx_range
            out.append(state.narrow(ax, k0, k1 - k0).contiguous())
        return out

    def gather(self, shards):
        """The whole-problem tensor from every rank's shard (every rank in
        this process)."""
        import torch

        if len(shards) != self.nranks:
            raise ValueError("gather needs every rank's shard in this process")
        return torch.cat(list(shards), dim=self.kx_axis())

    # -- the flow interface over sharded states ----------------------------------
    def _new(self):
        return [f._new() for f in self.flows]

    def get_rhs(self, states, out=None):
        out = self._new() if out is None else out
        for phase in range(3):
            if phase:
                self.comm.barrier()
            for f, s, o in zip(self.flows, states, out):
                f.rhs_phase(s, o, phase)
        return out

    def predict(self, states, rhs):
        return [f.predict(s, r) for f, s, r in zip(self.flows, states, rhs)]

    def _total(self, shares, err):
        """err[0] := sqrt(sum over every rank of the squared-norm shares)."""
        import torch

        acc = shares[0].clone()
        for sh in shares[1:]:
            acc += sh
        self.comm.sum_(acc)
        torch.sqrt(acc, out=err)
        return err

    def correct_fused(self, state_prev, prediction, rhs_prev, rhs_next, err, out=None):
        import torch

        out = prediction if out is None else out
        shares = [torch.empty(1, dtype=torch.float64, device=self.device) for _ in self.flows]
        res = [f.correct_fused(sp, p, rp, rn, sh, out=o)
               for f, sp, p, rp, rn, sh, o in zip(self.flows, state_prev, prediction,
                                                  rhs_prev, rhs_next, shares, out)]
        self._total(shares, err)
        return res

    def norm(self, v, out=None):
        import torch

        out = torch.empty(1, dtype=torch.float64, device=self.device) if out is None else out
        return self._total([f.norm(x) for f, x in zip(self.flows, v)], out)

    def correct_velocity(self, states):
        return [f.correct_velocity(s)[0] for f, s in zip(self.flows, states)], None

    def make_stepper(self, fused: bool = True):
        """predict_and_correct / iterate_correction over sharded states with
        the fused corrector (timestep.make_fused_stepper's contract)."""
        import torch

        def _err():
            return torch.empty(1, dtype=torch.float64, device=self.device)

        def predict_and_correct(states):
            rhs_prev = self.get_rhs(states)
            prediction = self.predict(states, rhs_prev)
            rhs_next = self.get_rhs(prediction)
            err = _err()
            prediction = self.correct_fused(states, prediction, rhs_prev, rhs_next, err,
                                            out=prediction)
            return prediction, rhs_next, err

        def iterate_correction(state_prev, prediction, rhs_prev):
            rhs_next = self.get_rhs(prediction)
            err = _err()
            prediction = self.correct_fused(state_prev, prediction, rhs_prev, rhs_next, err,
                                            out=prediction)
            return prediction, rhs_next, err

        return predict_and_correct, iterate_correction

    def get_stats(self, states) -> dict:
        """The flow's get_stats over every rank: each rank's sums
        (stats_sums), added over the ranks, then the reference's formulas."""
        import torch

        tot = None
        for f, st in zip(self.flows, states):
            sh = torch.tensor(f.stats_sums(st), dtype=torch.float64, device=self.device)
            tot = sh if tot is None else tot + sh
        self.comm.sum_(tot)
        return self.flows[0].stats_from_sums(tuple(float(v) for v in tot.tolist()))
