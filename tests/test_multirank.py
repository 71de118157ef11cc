"""Replica runs on N GPUs (bench.py --gpus N under torchrun): the path has no
data-path exchange, so the only multi-rank logic is the barrier and the job
step time as the maximum over ranks.  Exercised here with 2 gloo ranks on CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    import sys
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        dist.barrier()
        out[rank] = bench.max_over_ranks(1.5 + rank, "cpu")
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_step_time_is_the_max_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    port = _free_port()
    with ctx.Manager() as m:
        out = m.dict()
        procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
            assert p.exitcode == 0
        assert dict(out) == {0: 2.5, 1: 2.5}
