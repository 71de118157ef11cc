"""Point-sharded field evaluation over the ranks of a torch.distributed group.

Observation points are independent, so N GPUs evaluate a field N times
faster without any exchange while they compute: rank r takes the r-th
contiguous slice of the points (sizes differ by at most one), evaluates the
field of the whole geometry there with the device kernels, and one
all_gather (3 doubles per point, over NCCL on GPUs, gloo on CPU) gives every
rank the full result.  The geometry is replicated, which is what the field
path needs anyway: every point sees every source.

``relax_rows`` splits the relaxation itself: rank r holds the rows of its
contiguous slice of the elements (a row block of the interaction matrix,
radb200_intrc_create_rows), so a system too large for one device's memory,
or one that should relax faster, spreads over the ranks.  Each iteration is
the Jacobi + Anderson iteration of radb200_relax (RADB200_RLX_JACOBI): every
rank computes the proposal of its rows from the full magnetization
(radb200_relax_rows_step), one all_gather gives every rank the full residual
and one all_reduce the misfit, and the Anderson update of the full vector,
identical on every rank, yields the next magnetization.  That is the one real
exchange of the iteration: N M needs all of M on every row.
"""
from __future__ import annotations

import ctypes as C
import math
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


# ---------------------------------------------------------------------------
# row-block relaxation
# ---------------------------------------------------------------------------
class RowBlock:
    """Rows [e0, e1) of the interaction of a relaxation pack on this rank's
    device (radb200_intrc_create_rows); step() is radb200_relax_rows_step on
    torch tensors (float64, on the device)."""

    def __init__(self, pack, e0: int, e1: int, storage: int = 1):
        import torch
        self.pack, self.e0, self.e1 = pack, int(e0), int(e1)
        self._g = _native.GeomHolder(pack.elems)
        self._r = _native.RelaxHolder(pack.elem_src, pack.mat_kind, pack.mat, pack.mh)
        self._x = _native.GeomHolder(pack.ext) if pack.ext is not None else None
        h = C.c_int64(0)
        xg = C.cast(self._x.ptr, C.c_void_p) if self._x else None
        _native.check(_native.lib().radb200_intrc_create_rows(C.cast(self._g.ptr, C.c_void_p), C.cast(self._r.ptr, C.c_void_p),
                                                              xg, int(storage), self.e0, self.e1, C.byref(h)),
                      "radb200_intrc_create_rows")
        self.handle = h.value
        dev = torch.device("cuda", torch.cuda.current_device())
        m = 3 * (self.e1 - self.e0)
        self.Mp = torch.zeros(m, dtype=torch.float64, device=dev)
        self.F = torch.zeros(m, dtype=torch.float64, device=dev)
        self.H = torch.zeros(m, dtype=torch.float64, device=dev)

    def __call__(self, M, prec: float):
        sq = C.c_double(0.0)
        M = M.contiguous()
        _native.check(_native.lib().radb200_relax_rows_step(self.handle, M.data_ptr(), float(prec), self.Mp.data_ptr(),
                                                            self.F.data_ptr(), self.H.data_ptr(), C.byref(sq)),
                      "radb200_relax_rows_step")
        return self.Mp, self.F, self.H, float(sq.value)

    def free(self):
        if self.handle:
            _native.lib().radb200_intrc_free(self.handle)
            self.handle = 0

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


ANDERSON_DEPTH = 6


def relax_rows(pack, prec: float = 1e-10, max_iter: int = 1000, storage: int = 1, omega: float = 1.0,
               group=None, row_step: Optional[Callable] = None):
    """Relax the elements of pack (model.pack_interaction) with the
    interaction rows split over the ranks of group.  Returns (M [3n] as a
    numpy array, identical on every rank, and the status [misfit, max |M|,
    max |H|, iterations] of radb200_relax).

    row_step(e0, e1) -> callable(M, prec) returning (Mp_rows, F_rows,
    H_rows, sum |F_e|^2) for the rows [e0, e1) makes the device row block
    replaceable, so that the exchange and the Anderson iteration can be
    exercised without a GPU; it defaults to RowBlock."""
    import torch
    import torch.distributed as dist

    n = int(pack.elem_src.shape[0])
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    gloo = dist.get_backend(group) != "nccl"
    e0, e1 = shard_bounds(n, world, rank)
    if e1 <= e0:
        raise ValueError("more ranks than elements")
    step = (row_step or (lambda a, b: RowBlock(pack, a, b, storage)))(e0, e1)
    dev = torch.device("cpu") if row_step is not None else torch.device("cuda", torch.cuda.current_device())
    cdev = torch.device("cpu") if gloo else dev  # where the collectives run
    m = 3 * ((n + world - 1) // world)
    bounds = [shard_bounds(n, world, r) for r in range(world)]

    def gather(rows):
        buf = torch.zeros(m, dtype=torch.float64, device=cdev)
        buf[:rows.numel()] = rows.to(cdev)
        parts = [torch.empty_like(buf) for _ in range(world)]
        dist.all_gather(parts, buf, group=group)
        return torch.cat([parts[r][:3 * (b - a)] for r, (a, b) in enumerate(bounds)]).to(dev)

    def reduce(x, op):
        t = torch.tensor([x], dtype=torch.float64, device=cdev)
        dist.all_reduce(t, op=op, group=group)
        return float(t.item())

    M = torch.as_tensor(np.ascontiguousarray(pack.mat[:, 9:12]).reshape(-1), dtype=torch.float64).to(dev)
    AM = ANDERSON_DEPTH
    dX = torch.zeros((AM, 3 * n), dtype=torch.float64, device=dev)
    dF = torch.zeros_like(dX)
    Xprev = torch.zeros(3 * n, dtype=torch.float64, device=dev)
    Fprev = torch.zeros_like(Xprev)
    G = np.zeros((AM, AM))
    om = omega if 0.0 < omega <= 1.0 else 1.0
    misfit, best = math.inf, math.inf
    hist = head = 0
    have_prev = False
    it = 0
    hmax_local = 0.0
    try:
        for it in range(1, max_iter + 1):
            Mp_r, F_r, H_r, sq = step(M, prec)
            hmax_local = float(torch.linalg.vector_norm(H_r.reshape(-1, 3), dim=1).max()) if H_r.numel() else 0.0
            misfit = math.sqrt(reduce(sq, dist.ReduceOp.SUM) / n)
            if not math.isfinite(misfit):
                raise RuntimeError("relaxation produced a non-finite misfit")
            F = gather(F_r)
            if misfit <= prec:
                M = gather(Mp_r)  # accept the converged proposal
                break
            if misfit < best:
                best = misfit
            elif misfit > 4.0 * best:  # divergence guard: drop the history, damp harder
                hist = head = 0
                have_prev = False
                om = max(0.05, 0.5 * om)
            if have_prev:
                new = head
                dX[new] = M - Xprev
                dF[new] = F - Fprev
                head = (head + 1) % AM
                hist = min(hist + 1, AM)
                slots = [(new - k + AM) % AM for k in range(hist)]
                S = torch.stack([dF[s] for s in slots])
                gr = (S @ dF[new]).cpu().numpy()
                rhs = (S @ F).cpu().numpy()
                for k, s_ in enumerate(slots):
                    G[new, s_] = G[s_, new] = gr[k]
                A = G[np.ix_(slots, slots)].copy()
                A[np.diag_indices(hist)] += 1e-10 * max(G[s_, s_] for s_ in slots) + 1e-300
                Xprev, Fprev = M.clone(), F.clone()
                try:
                    gam = torch.as_tensor(np.linalg.solve(A, rhs), dtype=torch.float64, device=dev)
                    Xs = torch.stack([dX[s] for s in slots])
                    M = M + om * F - gam @ (Xs + om * S)
                except np.linalg.LinAlgError:
                    M = M + om * F
            else:
                Xprev, Fprev = M.clone(), F.clone()
                have_prev = True
                M = M + om * F
        Mh = M.cpu().numpy()
        st = np.array([misfit, float(np.linalg.norm(Mh.reshape(-1, 3), axis=1).max()),
                       reduce(hmax_local, dist.ReduceOp.MAX), float(min(it, max_iter))])
        return Mh, st
    finally:
        if hasattr(step, "free"):
            step.free()
