"""Multi-rank replica logic on CPU with the gloo backend (world size 2)."""

import os

import torch.multiprocessing as mp


def _worker(rank, world, port, out):
    import torch.distributed as dist

    from dnsjax_b200.replicas import max_over_ranks, replica_seed, total_steps

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = 10.0 + 5.0 * rank
        out[rank] = (max_over_ranks(ms, dist), replica_seed(4, rank),
                     total_steps(3, world))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_max_and_seeds():
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
    assert out[0][0] == out[1][0] == 15.0
    assert {out[0][1], out[1][1]} == {4, 5}
    assert out[0][2] == 6


def test_no_group_is_identity():
    from dnsjax_b200.replicas import max_over_ranks

    assert max_over_ranks(3.5) == 3.5
