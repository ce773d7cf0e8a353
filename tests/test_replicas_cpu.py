"""The multi-GPU form of the bench is N independent replicas (the path is kept on one GPU,
no sharding): the host logic of that form on two gloo ranks on the CPU.  The step time
reported is the largest over the ranks, every rank takes part in the same collective, and
the reference arm runs on rank 0 only."""
import io
import os
import sys
from contextlib import redirect_stdout

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        vals = bench.max_over_ranks([10.0 + rank, 5.0 - rank, 7.0 * (rank + 1)], dist, torch, "cpu")
        buf = io.StringIO()
        with redirect_stdout(buf):
            r = bench.reference_arm(None, rank, world) if rank != 0 else None
        out.put((rank, vals, r, buf.getvalue()))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_rank0_only_reference_arm():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = 29500 + os.getpid() % 2000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = {}
    for _ in procs:
        rank, vals, r, printed = out.get(timeout=120)
        res[rank] = (vals, r, printed)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank in (0, 1):
        assert res[rank][0] == [11.0, 5.0, 14.0]
    assert res[1][2] == ""        # rank 1 of the reference arm does no work and prints nothing
