"""CPU restatement of the adjoint of Radia's relaxation and field operator.

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the device
adjoint.  The product package never imports this module.

Forward problem (element frames, as assembled by the reference,
radintrc.cpp:831-877): M solves M = M_mat(H_ext + N M).  For a loss L(B(pts))
the gradient with respect to element parameters p is

    dL/dp = W.dB/dp|_M + lambda^T D (dH_ext/dp + dN/dp M) + lambda^T dM_mat/dp|_H,
    (I - D N)^T lambda = (dB/dM)^T W,   D = dM/dH (radmater.cpp:206-277),

with W = dL/dB.  Everything here is numpy on top of the C oracle: N and H_ext
from orc_assemble / orc_extfield, dB/dM by unit-magnetization field calls,
D from orc_material_dmdh, and dN/dp from full 3x3x3 derivative tensors of the
cuboid tensor Q (radrec.cpp:115-283):

    Q_aa = 1/(4 pi) sum_corners p atan(.)     Q_ab = -1/(4 pi) sum_corners p log(.)

whose derivatives are the corner sums in ``cuboid_dQ`` (checked against
central differences of the oracle field by tests/test_adjoint.py).
"""
from __future__ import annotations

import numpy as np

from . import oracle as O

C4PI = 1.0 / (4.0 * np.pi)
_PAIRS = [(0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)]


def _corner_partials(X, Y, Z):
    """d/dX, d/dY, d/dZ of the six corner functions (xx, yy, zz, xy, xz, yz):
    atan(YZ/(XR)), atan(XZ/(YR)), atan(XY/(ZR)), log(Z+R), log(Y+R), log(X+R)."""
    R = np.sqrt(X * X + Y * Y + Z * Z)
    sxy, sxz, syz = X * X + Y * Y, X * X + Z * Z, Y * Y + Z * Z
    with np.errstate(divide="ignore", invalid="ignore"):
        izr = np.where(Z >= 0, 1.0 / (Z + R), (R - Z) / sxy)
        iyr = np.where(Y >= 0, 1.0 / (Y + R), (R - Y) / sxz)
        ixr = np.where(X >= 0, 1.0 / (X + R), (R - X) / syz)
        d = np.stack([
            np.stack([-Y * Z / R * (1 / sxz + 1 / sxy), X * Z / (R * sxy), X * Y / (R * sxz)], -1),
            np.stack([Y * Z / (R * sxy), -X * Z / R * (1 / syz + 1 / sxy), X * Y / (R * syz)], -1),
            np.stack([Y * Z / (R * sxz), X * Z / (R * syz), -X * Y / R * (1 / syz + 1 / sxz)], -1),
            np.stack([X / R * izr, Y / R * izr, 1 / R], -1),
            np.stack([X / R * iyr, 1 / R, Z / R * iyr], -1),
            np.stack([1 / R, Y / R * ixr, Z / R * ixr], -1),
        ], -2)
    bad = ~((sxy > 0) & (sxz > 0) & (syz > 0))
    d[bad] = 0.0
    return d  # [..., 6, 3]


def cuboid_dQ(q, hd):
    """dQ_ab/dq_k and dQ_ab/dh_k ([..., 3, 3, 3]) of a cuboid with half widths
    hd at q relative to its centre."""
    q = np.asarray(q, dtype=np.float64)
    dq6 = np.zeros(q.shape[:-1] + (6, 3))
    dh6 = np.zeros_like(dq6)
    for ex in (-1.0, 1.0):
        for ey in (-1.0, 1.0):
            for ez in (-1.0, 1.0):
                e = np.array([ex, ey, ez])
                p = ex * ey * ez
                d = _corner_partials(*np.moveaxis(q - e * hd, -1, 0))
                dq6 += p * d
                dh6 += p * d * (-e)
    sign = np.array([1, 1, 1, -1, -1, -1], dtype=np.float64)[:, None] * C4PI
    dq6 *= sign
    dh6 *= sign
    dQq = np.zeros(q.shape[:-1] + (3, 3, 3))
    dQh = np.zeros_like(dQq)
    for k, (a, b) in enumerate(_PAIRS):
        dQq[..., a, b, :] = dQq[..., b, a, :] = dq6[..., k, :]
        dQh[..., a, b, :] = dQh[..., b, a, :] = dh6[..., k, :]
    return dQq, dQh


def _trf(elems, t):
    r = elems["trf"][t]
    return r[0:9].reshape(3, 3), r[9:12], r[12:21].reshape(3, 3), r[21]


def _images(elems, kind, idx):
    if kind == 0:
        t0, nt = elems["rec_img"][idx]
    else:
        t0, nt = elems["poly_info"][idx][2:4]
    return range(int(t0), int(t0) + int(nt))


def with_magnetization(pack, M):
    """Copy of the element geometry with magnetization M [3n] (element frames)."""
    g = {k: v.copy() for k, v in pack.elems.items()}
    for e, (kind, idx) in enumerate(pack.elem_src):
        if kind == 0:
            g["rec"][idx, 6:9] = M[3 * e:3 * e + 3]
        else:
            g["poly"][idx, 3:6] = M[3 * e:3 * e + 3]
    return g


def field_of(pack, M, pts, what=0):
    """B (what 0) or H (what 1) at pts from the elements magnetized by M and the
    external sources."""
    B = O.field(with_magnetization(pack, M), pts, what)
    if pack.ext is not None:
        B = B + O.field(pack.ext, pts, what)
    return B


def field_operator_T(pack, pts, W, what=0):
    """(dB/dM)^T W by unit-magnetization field calls."""
    n = pack.elem_src.shape[0]
    g = np.zeros(3 * n)
    for e in range(n):
        for a in range(3):
            M = np.zeros(3 * n)
            M[3 * e + a] = 1.0
            g[3 * e + a] = np.sum(O.field(with_magnetization(pack, M), pts, what) * W)
    return g


def dmdh(pack, H):
    n = pack.elem_src.shape[0]
    return np.array([O.material_dmdh(pack, e, H[3 * e:3 * e + 3]) for e in range(n)])


def solve_newton(pack, N, Hext, M0=None, tol=1e-14, max_iter=60):
    """FP64 Newton on M = M_mat(H_ext + N M) with dense solves (small models)."""
    n = pack.elem_src.shape[0]
    M = np.zeros(3 * n) if M0 is None else M0.copy()
    for _ in range(max_iter):
        H = Hext + N @ M
        F = np.concatenate([O.material_m(pack, e, H[3 * e:3 * e + 3]) for e in range(n)]) - M
        if np.linalg.norm(F) <= tol * max(1.0, np.linalg.norm(M)):
            break
        D = dmdh(pack, H)
        J = -np.eye(3 * n)
        for e in range(n):
            J[3 * e:3 * e + 3, :] += D[e] @ N[3 * e:3 * e + 3, :]
        M = M - np.linalg.solve(J, F)
    return M


def _rect_terms(pack, M, X, U, j):
    """Pair sums over observers X (lab) with weights U for cuboid source j:
    returns (d/dc_j, d/dd_j, d/dX [nobs,3]) of sum_x U(x).B_j(x)."""
    kind, idx = pack.elem_src[j]
    r = pack.elems["rec"][idx]
    c, hd = r[0:3], 0.5 * r[3:6]
    m = M[3 * j:3 * j + 3]
    gc = np.zeros(3)
    gd = np.zeros(3)
    gx = np.zeros_like(X)
    for t in _images(pack.elems, kind, idx):
        Minv, V, F, _ = _trf(pack.elems, t)
        q = (X - V) @ Minv.T - c
        dQq, dQh = cuboid_dQ(q, hd)
        ut = U @ F  # F^T u per observer
        s_q = np.einsum("na,nabk,b->nk", ut, dQq, m)
        s_h = np.einsum("na,nabk,b->nk", ut, dQh, m)
        gc -= s_q.sum(0)
        gd += 0.5 * s_h.sum(0)
        gx += s_q @ Minv
    return gc, gd, gx


def gradients(pack, M, pts, W, what=0, fd_step_ext=1e-4):
    """dL/dMr, dL/dchi, dL/dc, dL/dd per element for L with dL/dB(pts) = W,
    at the converged magnetization M."""
    n = pack.elem_src.shape[0]
    N = O.assemble(pack)
    Hext = O.extfield(pack)
    H = Hext + N @ M
    D = dmdh(pack, H)
    gM = field_operator_T(pack, pts, W, what)
    A = np.eye(3 * n)
    for e in range(n):
        A[3 * e:3 * e + 3, :] -= D[e] @ N[3 * e:3 * e + 3, :]
    lam = np.linalg.solve(A.T, gM)
    # lab-frame observer weights u_e = rowT_e^T D_e^T lambda_e at the element centres
    X = np.zeros((n, 3))
    U = np.zeros((n, 3))
    Jobs = np.zeros((n, 3, 3))
    for e, (kind, idx) in enumerate(pack.elem_src):
        t0 = next(iter(_images(pack.elems, kind, idx)))
        Minv, V, F, s = _trf(pack.elems, t0)
        c = pack.elems["rec"][idx, 0:3] if kind == 0 else pack.elems["poly"][idx, 0:3]
        X[e] = F @ c / s + V
        Jobs[e] = F / s
        U[e] = (s * Minv).T @ (D[e].T @ lam[3 * e:3 * e + 3])
    gc = np.zeros((n, 3))
    gd = np.zeros((n, 3))
    gobs = np.zeros((n, 3))
    Wp = np.asarray(W, dtype=np.float64).reshape(-1, 3)
    P = np.asarray(pts, dtype=np.float64).reshape(-1, 3)
    for j, (kind, idx) in enumerate(pack.elem_src):
        if kind != 0:
            continue
        c1, d1, gx = _rect_terms(pack, M, X, U, j)   # through the solve
        c2, d2, _ = _rect_terms(pack, M, P, Wp, j)   # the loss field directly
        gc[j] += c1 + c2
        gd[j] += d1 + d2
        gobs += gx
    if pack.ext is not None:
        h = fd_step_ext
        for a in range(3):
            dx = np.zeros(3)
            dx[a] = h
            dH = (O.field(pack.ext, X + dx, 1) - O.field(pack.ext, X - dx, 1)) / (2 * h)
            gobs[:, a] += np.sum(U * dH, axis=1)
    for e, (kind, idx) in enumerate(pack.elem_src):
        if kind == 0:
            gc[e] += Jobs[e].T @ gobs[e]
    chi = np.zeros((n, 3, 3))
    for e in range(n):
        if pack.mat_kind[e] == 0:
            chi[e] = np.outer(lam[3 * e:3 * e + 3], H[3 * e:3 * e + 3])
    return dict(lam=lam, gM=gM, Mr=lam.copy(), chi=chi.reshape(-1), c=gc.reshape(-1), d=gd.reshape(-1))
