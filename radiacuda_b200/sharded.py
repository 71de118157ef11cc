"""Point-sharded field evaluation over the ranks of a torch.distributed group.

Observation points are independent, so N GPUs evaluate a field N times
faster without any exchange while they compute: rank r takes the r-th
contiguous slice of the points (sizes differ by at most one), evaluates the
field of the whole geometry there with the device kernels, and one
all_gather (3 doubles per point, over NCCL on GPUs, gloo on CPU) gives every
rank the full result.  The geometry is replicated, which is what the field
path needs anyway: every point sees every source.

This is the point-sharded Fld of the multi-GPU plan; the dense interaction
matrix is not sharded (one B200 holds the 60,000^2 system of the largest
model in FP64 and FP32).
"""
from __future__ import annotations

from typing import Callable, Optional, Tuple

import numpy as np

from . import _native


def shard_bounds(n: int, world: int, rank: int) -> Tuple[int, int]:
    """[lo, hi) of rank's contiguous slice of n items; the first n % world
    ranks take one more."""
    q, r = divmod(int(n), int(world))
    lo = rank * q + min(rank, r)
    return lo, lo + q + (1 if rank < r else 0)


def field_sharded(geom, pts, what: int = 0, precision: int = 0, group=None,
                  point_field: Optional[Callable] = None) -> np.ndarray:
    """Field [n, 3] of the packed geometry at pts [n, 3] (what 0 B, 1 H, 2 M),
    this rank evaluating its slice and all ranks receiving the whole array.

    point_field(geom, pts, what, precision) evaluates one slice; it defaults
    to the device field (radb200_field) and is replaceable so that the
    sharding can be exercised without a GPU."""
    import torch
    import torch.distributed as dist

    P = np.ascontiguousarray(np.asarray(pts, dtype=np.float64).reshape(-1, 3))
    n = P.shape[0]
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    fn = point_field or _native.field
    lo, hi = shard_bounds(n, world, rank)
    local = fn(geom, P[lo:hi], what, precision) if hi > lo else np.zeros((0, 3))
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" else torch.device("cpu")
    m = (n + world - 1) // world
    buf = torch.zeros((max(m, 1), 3), dtype=torch.float64, device=dev)
    if hi > lo:
        buf[:hi - lo] = torch.from_numpy(np.ascontiguousarray(local, dtype=np.float64)).to(dev)
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    out = np.empty((n, 3))
    for r, t in enumerate(parts):
        a, b = shard_bounds(n, world, r)
        if b > a:
            out[a:b] = t[:b - a].cpu().numpy()
    return out


def Fld(obj: int, fid: str, pts, group=None, precision: str = "double") -> np.ndarray:
    """rad.Fld over the ranks of group for an [n, 3] array of points: the
    same columns as rad.Fld's array form (e.g. 'bxbz' -> [n, 2], 'b' -> [n, 3]),
    on every rank."""
    from . import rad
    from .model import pack_sources

    parts = rad._parse_id(fid)
    prec = {"double": 0, "single": 1, "fast": 2}.get(str(precision).lower())
    if prec is None:
        raise rad.RadiaError("Radia::Error000: precision must be 'double', 'single' or 'fast'")
    geom = pack_sources(rad._objs, int(obj), tuple(rad._rand))
    vals = {w: field_sharded(geom, pts, {"b": 0, "h": 1, "m": 2}[w], prec, group)
            for w in sorted({p[0] for p in parts})}
    cols = [vals[ch] if comp is None else vals[ch][:, comp:comp + 1] for ch, comp in parts]
    return cols[0] if len(cols) == 1 else np.concatenate(cols, axis=1)
