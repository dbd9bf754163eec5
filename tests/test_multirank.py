"""The multi-rank path of bench.py on CPU: two gloo ranks (world_size 2), as
torchrun launches them. Each rank assembles its own replica (the path has no
exchange step); the job time is the maximum over the ranks of the per-rank
device time, and every rank takes the same collective steps."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        import bench
        local = [12.5, 20.0][rank]
        out[rank] = bench.job_ms(local, world, torch.device("cpu"))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_job_time_is_max_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    assert out[0] == out[1] == 20.0


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.job_ms(7.0, 1, None) == 7.0
