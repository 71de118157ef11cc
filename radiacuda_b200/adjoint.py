"""Gradients of field losses through the device relaxation.

``FieldProblem`` holds a Radia model (built with ``radiacuda_b200.rad``), a
fixed set of field points and the solver settings.  Its forward pass maps the
per-element parameters

    mr     [n, 3]     remanence of each relaxable element's material
    chi    [n, 3, 3]  susceptibility tensor (linear elements; ignored otherwise)
    centre [n, 3]     centre of each rectangular element
    dims   [n, 3]     full widths of each rectangular element

(all in each element's object frame) to B or H at the points: device
assembly, the solve (dense direct solve for linear models, Newton-Krylov
relaxation otherwise) and the device field.  Its backward pass is the
hand-written adjoint of the library (radb200_field_vjp, radb200_adjoint_solve,
radb200_adjoint_grad): one transposed solve with dM/dH at the converged state
and pair-wise derivative contractions, never a materialised dN/dp.

``relaxed_field`` wraps the two passes in a ``torch.autograd.Function`` so a
loss written in torch (per-block parameters mapped to elements with
``FieldProblem.elements_of``, easy-axis susceptibilities with
``FieldProblem.aniso_chi``) differentiates end to end.

No counterpart in the reference: Radia has no derivatives.
"""
from __future__ import annotations

import time
import warnings
from typing import Dict, Optional, Sequence

import numpy as np

from . import _native, model
from . import rad as _rad

_WHAT = {"b": 0, "h": 1}


class FieldProblem:
    def __init__(self, obj: int, pts, what: str = "b", srcobj: int = 0, storage: int = 1,
                 solver: str = "auto", prec: float = 1e-13, max_iter: int = 2000, adj_rtol: float = 1e-12):
        if what not in _WHAT:
            raise ValueError("what must be 'b' or 'h'")
        self.pack = model.pack_interaction(_rad._objs, int(obj), int(srcobj), tuple(_rad._rand))
        self.pts = np.ascontiguousarray(np.asarray(pts, dtype=np.float64).reshape(-1, 3))
        self.what = _WHAT[what]
        self.storage = storage
        linear = bool(np.all(self.pack.mat_kind == 0))
        self.solver = ("direct" if linear else "newton") if solver == "auto" else solver
        self.prec, self.max_iter, self.adj_rtol = prec, max_iter, adj_rtol
        self.n = self.pack.elem_src.shape[0]
        e = self.pack.elems
        self.rect = self.pack.elem_src[:, 0] == 0
        idx = self.pack.elem_src[:, 1]
        self.centre0 = np.zeros((self.n, 3))
        self.dims0 = np.zeros((self.n, 3))
        self.centre0[self.rect] = e["rec"][idx[self.rect], 0:3]
        self.dims0[self.rect] = e["rec"][idx[self.rect], 3:6]
        self.mr0 = self.pack.mat[:, 9:12].copy()
        self.chi0 = self.pack.mat[:, 0:9].reshape(-1, 3, 3).copy()
        self._intrc: Optional[_native.NativeInteraction] = None
        self._M: Optional[np.ndarray] = None
        self.last_status: Dict[str, np.ndarray] = {}
        self.last_timing: Dict[str, float] = {}   # wall seconds of each phase of the last passes

    # ---- parameter helpers -------------------------------------------------
    def elements_of(self, handle: int) -> np.ndarray:
        """Indices of the relaxable elements that lie under object ``handle``."""
        leaves = {lf.handle for lf in model.collect_leaves(_rad._objs, int(handle))}
        return np.array([e for e, lf in enumerate(self.pack.leaves) if lf.handle in leaves], dtype=np.int64)

    def linear_ksi(self) -> np.ndarray:
        """(ksi_par, ksi_perp) of each element's linear material (NaN otherwise)."""
        out = np.full((self.n, 2), np.nan)
        for e, lf in enumerate(self.pack.leaves):
            m = lf.obj.mat
            if m.kind == 0:
                out[e] = m.ksi
        return out

    @staticmethod
    def aniso_chi(mr, ksi):
        """chi = ksi_perp I + (ksi_par - ksi_perp) L L^T, L = mr/|mr|
        (radTLinearAnisotropMaterial, radmater.h:292-303); torch or numpy."""
        try:
            import torch
            if isinstance(mr, torch.Tensor):
                ksi_t = torch.as_tensor(ksi, dtype=mr.dtype, device=mr.device)
                L = mr / torch.linalg.norm(mr, dim=-1, keepdim=True)
                eye = torch.eye(3, dtype=mr.dtype, device=mr.device)
                return ksi_t[:, 1, None, None] * eye + (ksi_t[:, 0] - ksi_t[:, 1])[:, None, None] * L[:, :, None] * L[:, None, :]
        except ImportError:
            pass
        mr = np.asarray(mr, dtype=np.float64)
        L = mr / np.linalg.norm(mr, axis=-1, keepdims=True)
        return ksi[:, 1, None, None] * np.eye(3) + (ksi[:, 0] - ksi[:, 1])[:, None, None] * L[:, :, None] * L[:, None, :]

    # ---- passes (numpy) ----------------------------------------------------
    def _apply(self, mr, chi, centre, dims):
        p = self.pack
        p.mat[:, 9:12] = mr
        lin = p.mat_kind == 0
        p.mat[lin, 0:9] = np.asarray(chi).reshape(-1, 9)[lin]
        idx = p.elem_src[:, 1]
        p.elems["rec"][idx[self.rect], 0:3] = np.asarray(centre)[self.rect]
        p.elems["rec"][idx[self.rect], 3:6] = np.asarray(dims)[self.rect]

    def forward(self, mr=None, chi=None, centre=None, dims=None) -> np.ndarray:
        self._apply(self.mr0 if mr is None else mr, self.chi0 if chi is None else chi,
                    self.centre0 if centre is None else centre, self.dims0 if dims is None else dims)
        if self._intrc is not None:
            self._intrc.free()
        t0 = time.perf_counter()
        I = _native.NativeInteraction(self.pack, storage=self.storage)
        t1 = time.perf_counter()
        if self.solver == "direct":
            M, st = I.direct(0 if self.storage == 1 else 1, self.prec, self.max_iter)
        else:
            M, _, st = I.relax(1 if self.solver == "newton" else 0, self.prec, self.max_iter, True, 1.0,
                               np.zeros(3 * self.n))
        self._intrc, self._M = I, M
        self.last_status["forward"] = st
        if not st[0] <= self.prec:
            # the reference's wording for a relaxation that stopped short
            warnings.warn("The specified accuracy was not reached. This may indicate diverging or incomplete "
                          f"relaxation (misfit {st[0]:.3e}).", RuntimeWarning)
        t2 = time.perf_counter()
        g = {k: v.copy() for k, v in self.pack.elems.items()}
        for e, (kind, idx) in enumerate(self.pack.elem_src):
            if kind == 0:
                g["rec"][idx, 6:9] = M[3 * e:3 * e + 3]
            else:
                g["poly"][idx, 3:6] = M[3 * e:3 * e + 3]
        F = _native.field(g, self.pts, self.what, 0)
        if self.pack.ext is not None:
            F = F + _native.field(self.pack.ext, self.pts, self.what, 0)
        t3 = time.perf_counter()
        self.last_timing.update(assembly=t1 - t0, solve=t2 - t1, field=t3 - t2)
        return F

    def backward(self, W) -> Dict[str, np.ndarray]:
        """Gradients of sum(W * F) w.r.t. mr, chi, centre, dims at the last forward."""
        if self._intrc is None:
            raise RuntimeError("backward before forward")
        I = self._intrc
        W = np.ascontiguousarray(np.asarray(W, dtype=np.float64).reshape(-1, 3))
        t0 = time.perf_counter()
        gM, gc, gd = I.field_vjp(self._M, self.pts, self.what, W)
        t1 = time.perf_counter()
        lam, st = I.adjoint_solve(gM, self.adj_rtol, 500)
        t2 = time.perf_counter()
        self.last_status["adjoint"] = st
        g = I.adjoint_grad(lam)
        t3 = time.perf_counter()
        self.last_timing.update(field_vjp=t1 - t0, adjoint_solve=t2 - t1, adjoint_grad=t3 - t2)
        return dict(mr=g["Mr"].reshape(-1, 3), chi=g["chi"].reshape(-1, 3, 3),
                    centre=(g["c"] + gc).reshape(-1, 3), dims=(g["d"] + gd).reshape(-1, 3))

    @property
    def magnetization(self) -> Optional[np.ndarray]:
        return None if self._M is None else self._M.reshape(-1, 3)


def relaxed_field(problem: FieldProblem, mr, chi, centre, dims):
    """torch.autograd.Function over FieldProblem: returns F [npts, 3] (float64)."""
    import torch

    class _RelaxedField(torch.autograd.Function):
        @staticmethod
        def forward(ctx, mr_, chi_, centre_, dims_):
            F = problem.forward(*(t.detach().cpu().double().numpy() for t in (mr_, chi_, centre_, dims_)))
            ctx.dev = mr_.device
            return torch.from_numpy(F).to(mr_.device)

        @staticmethod
        def backward(ctx, gF):
            g = problem.backward(gF.detach().cpu().double().numpy())
            return tuple(torch.from_numpy(g[k]).to(ctx.dev) for k in ("mr", "chi", "centre", "dims"))

    return _RelaxedField.apply(mr, chi, centre, dims)
