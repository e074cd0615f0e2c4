"""CPU: the multi-rank plumbing of bench.py with two gloo ranks — the batch is
sharded as replicas (no data-path collective); the only collective is the
max-over-ranks reduction of the timed region, and only rank 0 runs the
reference arm."""
import datetime
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import torch.distributed as dist

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench

    w, r, l = bench.dist_setup()
    v = bench.max_over_ranks(1.5 + rank, world)

    class Args:
        steps, warmup, gpus = 1, 0, world

    # rank != 0 returns at once from the reference arm (nothing printed, no work)
    ref = bench.run_reference(Args, world, rank) if rank != 0 else None
    q.put((rank, w, r, l, v, ref))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[:4] for o in out] == [(0, 2, 0, 0), (1, 2, 1, 1)]
    assert all(o[4] == 2.5 for o in out)  # max over ranks
    assert out[1][5] is None
