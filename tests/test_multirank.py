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


def _shard_main(rank, world, port, out):
    import sys
    import datetime

    import numpy as np
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "tests"))
    import models as MD
    import oracle.oracle as O
    from radiacuda_b200 import model, rad, sharded
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        h = MD.mixed_sym(rad)
        g = model.pack_sources(rad._objs, h, tuple(rad._rand))
        P = np.random.default_rng(8).uniform(-80, 90, size=(1001, 3)) + 0.0137
        calls = []

        def oracle_slice(geom, pts, what, precision):
            calls.append(pts.shape[0])
            return O.field(geom, pts, what)

        got = sharded.field_sharded(g, P, 0, 0, point_field=oracle_slice)
        out[rank] = (bool(np.array_equal(got, O.field(g, P, 0))), calls)
    finally:
        dist.destroy_process_group()


def test_point_sharded_field_over_three_gloo_ranks():
    """Each rank evaluates its contiguous slice (1001 points: 334, 334, 333)
    and all ranks end with the whole field, identical to one evaluation."""
    from radiacuda_b200.sharded import shard_bounds
    assert [shard_bounds(1001, 3, r) for r in range(3)] == [(0, 334), (334, 668), (668, 1001)]
    assert shard_bounds(2, 3, 2) == (2, 2)
    ctx = mp.get_context("spawn")
    port = _free_port()
    with ctx.Manager() as m:
        out = m.dict()
        procs = [ctx.Process(target=_shard_main, args=(r, 3, port, out)) for r in range(3)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=180)
            assert p.exitcode == 0
        res = dict(out)
    assert all(res[r][0] for r in range(3))
    assert [res[r][1] for r in range(3)] == [[334], [334], [333]]


def _nccl_main(port, out):
    import sys
    import datetime

    import numpy as np
    import torch
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "tests"))
    import models as MD
    from radiacuda_b200 import rad, sharded
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60))
    try:
        h = MD.mixed_sym(rad)
        P = np.random.default_rng(8).uniform(-80, 90, size=(4097, 3)) + 0.0137
        a = sharded.Fld(h, "bxbzh", P)
        b = rad.Fld(h, "bxbzh", P)
        out[0] = bool(np.array_equal(a, b)) and a.shape == (4097, 5)
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
def test_sharded_fld_over_nccl_equals_fld(cuda):
    """The sharded Fld through a one-rank NCCL group on the GPU returns what
    rad.Fld returns (the multi-GPU runs of this pool have one GPU)."""
    ctx = mp.get_context("spawn")
    port = _free_port()
    with ctx.Manager() as m:
        out = m.dict()
        p = ctx.Process(target=_nccl_main, args=(port, out))
        p.start()
        p.join(timeout=300)
        assert p.exitcode == 0
        assert out[0]


def _utimpi_main(rank, world, port, out):
    import sys
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from radiacuda_b200 import rad
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        res = {"on": rad.UtiMPI("on"), "barrier": rad.UtiMPI("barrier")}
        mine = [[10.0 * rank, 1.0], [2.0]]
        res["all"] = rad.UtiMPI("share", mine, 1)
        res["to0"] = rad.UtiMPI("share", mine, 1, 0)
        res["off"] = rad.UtiMPI("off")
        out[rank] = res
    finally:
        dist.destroy_process_group()


def test_utimpi_over_two_gloo_ranks():
    """rad.UtiMPI on the default group: the rank, a barrier, and 'share' from
    rank 1 to every rank and to rank 0 only (data flattened to floats)."""
    ctx = mp.get_context("spawn")
    port = _free_port()
    with ctx.Manager() as m:
        out = m.dict()
        procs = [ctx.Process(target=_utimpi_main, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
            assert p.exitcode == 0
        res = dict(out)
    for r in (0, 1):
        assert res[r]["on"] == r and res[r]["barrier"] == r and res[r]["off"] == r
        assert res[r]["all"] == [10.0, 1.0, 2.0]
    assert res[0]["to0"] == [10.0, 1.0, 2.0]
    assert res[1]["to0"] == [10.0, 1.0, 2.0]


def _utimpi_partial_main(rank, world, port, out):
    import sys
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from radiacuda_b200 import rad
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        res = {}
        # broadcast from rank 2: the receivers pass no data but still join
        res["bcast"] = rad.UtiMPI("share", [[7.0, 8.0]] if rank == 2 else None, 2)
        # point to point from rank 1 to rank 0: rank 2 does not call share at all
        if rank in (0, 1):
            res["p2p"] = rad.UtiMPI("share", [[1.5 + rank, 2.5]] if rank == 1 else None, 1, 0)
        res["barrier"] = rad.UtiMPI("barrier")
        out[rank] = res
    finally:
        dist.destroy_process_group()


def test_utimpi_share_with_receivers_without_data_over_three_gloo_ranks():
    """'share' as the reference's MPI share: receivers that pass no data join
    the broadcast and get their rank back; a rankTo >= 0 share involves only
    the sending and the receiving rank."""
    ctx = mp.get_context("spawn")
    port = _free_port()
    with ctx.Manager() as m:
        out = m.dict()
        procs = [ctx.Process(target=_utimpi_partial_main, args=(r, 3, port, out)) for r in range(3)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
            assert p.exitcode == 0
        res = dict(out)
    assert res[0]["bcast"] == 0 and res[1]["bcast"] == 1 and res[2]["bcast"] == [7.0, 8.0]
    assert res[1]["p2p"] == [2.5, 2.5]
    assert res[0]["p2p"] == 0
    assert "p2p" not in res[2]
    assert [res[r]["barrier"] for r in range(3)] == [0, 1, 2]


def test_utimpi_without_a_process_group(rad):
    assert rad.UtiMPI("on") == 0 and rad.UtiMPI("barrier") == 0 and rad.UtiMPI("off") == 0
    assert rad.UtiMPI("share", [[1, 2], [3]]) == [1.0, 2.0, 3.0]
    with pytest.raises(RuntimeError, match="Error000"):
        rad.UtiMPI("start")
