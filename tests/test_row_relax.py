"""Row-block relaxation over ranks (radiacuda_b200.sharded.relax_rows).

CPU (gloo, spawned ranks): the exchange and the Anderson iteration of the
driver, with each rank's device row block replaced by the oracle's proposal
for the same rows (the oracle's interaction matrix, the per-element implicit
solve done exactly); runs on 1, 2 and 3 ranks must agree with each other, and
the linear model with the oracle's dense solve.

GPU: the device row blocks (radb200_intrc_create_rows / relax_rows_step) of
one rank against radb200_relax on the whole interaction, and 2 gloo ranks
sharing the device (the ranks exchange through the host; no kernel of one
waits on the other) against 1.
"""
import datetime
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _model(rad, which):
    import models as MD
    from radiacuda_b200 import model
    if which == "linear":
        h = MD.sym_blocks(rad, div=2)
    else:
        h = MD.hybrid_undulator(rad, n_pairs=2, pole_div=(2, 1, 2), block_div=(2, 1, 1))[0]
    return model.pack_interaction(rad._objs, h, 0, tuple(rad._rand))


def oracle_rows(pack):
    """row_step for relax_rows from the oracle: the proposal of rows [e0, e1)."""
    import torch

    from oracle import oracle as O
    N = O.assemble(pack)
    He = O.extfield(pack)

    def make(e0, e1):
        Hkeep = np.zeros(3 * (e1 - e0))  # each row's last field: the next solve's start

        def step(M, prec):
            Mn = M.cpu().numpy()
            Hall = N[3 * e0:3 * e1] @ Mn + He[3 * e0:3 * e1]
            Mp = np.zeros(3 * (e1 - e0))
            for e in range(e0, e1):
                s, r = slice(3 * e, 3 * e + 3), slice(3 * (e - e0), 3 * (e - e0) + 3)
                Q = N[s, s]
                Hq = Hall[r] - Q @ Mn[s]

                def res(H):
                    return H - Hq - Q @ O.material_m(pack, e, H)
                H = Hkeep[r].copy()
                F = res(H)
                for _ in range(100):  # Newton with backtracking on H - Hq - Q M(H) = 0
                    nf = np.linalg.norm(F)
                    if nf <= 1e-15 * max(1.0, np.linalg.norm(H)):
                        break
                    dH = np.linalg.solve(np.eye(3) - Q @ O.material_dmdh(pack, e, H), F)
                    lam = 1.0
                    while lam > 1e-6:
                        Ht = H - lam * dH
                        Ft = res(Ht)
                        if np.linalg.norm(Ft) < nf:
                            break
                        lam *= 0.5
                    if lam <= 1e-6:
                        break
                    H, F = Ht, Ft
                Hkeep[r] = H
                Mp[r] = O.material_m(pack, e, H)
            Hn = Hkeep.copy()
            F = Mp - Mn[3 * e0:3 * e1]
            t = lambda a: torch.from_numpy(np.ascontiguousarray(a))  # noqa: E731
            return t(Mp), t(F), t(Hn), float(np.sum(F * F))
        return step
    return make


def _rank_main(rank, world, port, which, out):
    sys.path[:0] = [ROOT, os.path.join(ROOT, "tests")]
    import torch.distributed as dist

    from radiacuda_b200 import rad, sharded
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        pack = _model(rad, which)
        M, st = sharded.relax_rows(pack, prec=1e-12, max_iter=2000, row_step=oracle_rows(pack))
        out[rank] = (M, st)
    finally:
        dist.destroy_process_group()


def _run(world, which):
    ctx = mp.get_context("spawn")
    port = _free_port()
    with ctx.Manager() as m:
        out = m.dict()
        procs = [ctx.Process(target=_rank_main, args=(r, world, port, which, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=300)
            assert p.exitcode == 0
        return [out[r] for r in range(world)]


@pytest.mark.parametrize("which", ["linear", "saturating"])
def test_row_relaxation_same_on_1_2_3_gloo_ranks(rad, which):
    from oracle import oracle as O
    res = {w: _run(w, which) for w in (1, 2, 3)}
    M1, st1 = res[1][0]
    assert st1[0] <= 1e-12, st1
    scale = np.abs(M1).max()
    for w in (2, 3):
        for M, st in res[w]:
            assert st[0] <= 1e-12, (w, st)
            # every rank holds the same full magnetization
            assert np.abs(M - res[w][0][0]).max() == 0.0
            assert np.abs(M - M1).max() <= 1e-11 * scale, w
    if which == "linear":
        pack = _model(rad, which)
        Md = O.linear_direct(pack, O.assemble(pack), O.extfield(pack))
        assert np.abs(M1 - Md).max() <= 1e-10 * scale


def test_row_bounds_cover_the_elements():
    from radiacuda_b200.sharded import shard_bounds
    for n in (1, 7, 640):
        for world in (1, 2, 3, 8):
            if world > n:
                continue
            b = [shard_bounds(n, world, r) for r in range(world)]
            assert b[0][0] == 0 and b[-1][1] == n
            assert all(b[r][1] == b[r + 1][0] for r in range(world - 1))
            assert max(y - x for x, y in b) - min(y - x for x, y in b) <= 1


# ---------------------------------------------------------------------------
# GPU
# ---------------------------------------------------------------------------
def _gpu_rank_main(rank, world, port, which, out):
    sys.path[:0] = [ROOT, os.path.join(ROOT, "tests")]
    import torch
    import torch.distributed as dist

    from radiacuda_b200 import rad, sharded
    torch.cuda.set_device(0)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        pack = _model(rad, which)
        M, st = sharded.relax_rows(pack, prec=1e-12, max_iter=2000, storage=1)
        out[rank] = (M, st)
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
@pytest.mark.parametrize("which", ["linear", "saturating"])
def test_device_row_blocks_match_whole_interaction(cuda, rad, which):
    from radiacuda_b200 import _native
    pack = _model(rad, which)
    I = _native.NativeInteraction(pack, storage=1)
    Mw, _, stw = I.relax(0, 1e-12, 2000, True, 1.0, np.zeros(3 * pack.elem_src.shape[0]))
    I.free()
    assert stw[0] <= 1e-12
    ctx = mp.get_context("spawn")
    res = {}
    for world in (1, 2):
        port = _free_port()
        with ctx.Manager() as m:
            out = m.dict()
            procs = [ctx.Process(target=_gpu_rank_main, args=(r, world, port, which, out)) for r in range(world)]
            for p in procs:
                p.start()
            for p in procs:
                p.join(timeout=300)
                assert p.exitcode == 0
            res[world] = [out[r] for r in range(world)]
    scale = np.abs(Mw).max()
    for world, rr in res.items():
        for M, st in rr:
            assert st[0] <= 1e-12, (world, st)
            assert np.abs(M - Mw).max() <= 1e-10 * scale, world
    assert np.abs(res[2][0][0] - res[2][1][0]).max() == 0.0
