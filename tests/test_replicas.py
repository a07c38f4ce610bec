"""The multi-GPU path is N independent replicas (no collective on the data
path): the bench's rank context and whole-job aggregation, run as two CPU
ranks over gloo."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from cfdtest import ROOT


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out) -> None:
    import sys
    import datetime

    import torch
    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    ctx = bench.Ctx(torch, dist, world, rank, rank, device="cpu")
    ctx.barrier()
    # rank r processed (r + 1) * 1e9 cell updates in (r + 1) * 100 ms
    v = bench.job_throughput(ctx, (rank + 1) * 1e9, (rank + 1) * 100.0)
    reqs = bench.served_requests(6, bench.SEED + 7919 * rank)
    out.put((rank, ctx.max(rank * 2.0), ctx.sum(1.5), v, reqs))
    dist.destroy_process_group()


def test_two_replicas_aggregate_over_gloo():
    world, port = 2, _free_port()
    ctxm = mp.get_context("spawn")
    q = ctxm.Queue()
    procs = [ctxm.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, mx, sm, v, _ in res:
        assert mx == 2.0 and sm == 3.0
        # (1e9 + 2e9) updates over the slowest rank's 0.2 s
        assert v == pytest.approx(15.0)
    # each replica serves its own request stream
    assert res[0][4] != res[1][4]
