"""Radia-compatible Python API for the B200 relaxation hot path.

Function names, argument meanings, defaults, return shapes and error
behaviour follow the reference binding (cpp/src/clients/python/radpy.cpp,
method table :3341-3440) for the subset of Radia that builds and solves the
models of the hot path: magnetized cuboids and polyhedra, containers,
subdivision of cuboids, space transformations and symmetries, linear and
saturating materials, current arcs / racetracks / current blocks, background
fields, ``RlxPre`` / ``RlxAuto`` / ``Solve`` and ``Fld``.

Everything numeric runs on the GPU through libradb200 (include/radb200.h);
there is no CPU fallback -- a missing library or device raises.
"""
from __future__ import annotations

import io
import math
import pickle
from typing import Any, Dict, List, Optional, Sequence

import numpy as np

from . import _native, model
from .model import (ArcCur, Bckg, Container, InteractionPack, Material, Obj, Polyhedron, RadiaError,
                    RecMag, Trf, collect_leaves, images_of, pack_interaction, pack_sources, trf_field_inversion,
                    trf_plane_sym, trf_rotation, trf_translation)

__all__ = [
    "ObjRecMag", "ObjRecCur", "ObjPolyhdr", "ObjThckPgn", "ObjMltExtPgn", "ObjMltExtRtg", "ObjFullMag",
    "ObjCylMag", "ObjArcPgnMag", "ObjDrwAtr", "ObjDegFre", "ObjArcCur", "ObjRaceTrk", "ObjBckg",
    "ObjCnt", "ObjAddToCnt", "ObjCntStuf", "ObjCntSize", "ObjDivMag", "ObjM", "ObjSetM",
    "TrfTrsl", "TrfRot", "TrfPlSym", "TrfInv", "TrfCmbL", "TrfCmbR", "TrfMlt", "TrfOrnt",
    "TrfZerPara", "TrfZerPerp", "MatLin", "MatSatIsoFrm", "MatApl",
    "RlxPre", "RlxAuto", "Solve", "Fld", "FldLst", "FldInt", "FldPtcTrj", "FldCmpCrt", "FldCmpPrc", "FldLenRndSw", "FldLenTol",
    "UtiDel", "UtiDelAll", "UtiDmp", "UtiDmpPrs", "UtiMPI", "UtiVer", "UtiFldLastBackend", "UtiAsmLastBackend",
    "UtiGpuFallback",
]

# --------------------------------------------------------------------------
# global state (the reference keeps the same in radTApplication)
# --------------------------------------------------------------------------
_objs: Dict[int, Any] = {}
_next = [1]
# radTConvergRepair defaults (radcnvrg.h:37-45); FldLenRndSw('off') zeroes them
_rand_on = [1e-09, 1e-11, 1e-09]
_rand = list(_rand_on)
# radTCompCriterium defaults (cpp/src/core/radg3d.h:468-485); FldInt reads PrcBInt
_PRC_DEFAULT = {"PrcB": 1e-4, "PrcA": 1e-3, "PrcBInt": 1e-3, "PrcForce": 1.0, "PrcTorque": 10.0,
                "PrcEnergy": 10.0, "PrcCoord": -1.0, "PrcAngle": -1.0}
_prc = dict(_PRC_DEFAULT)
_last_fld = ["none"]
_last_asm = ["none"]
_fallback = ["cpu"]


def _add(o) -> int:
    h = _next[0]
    _next[0] += 1
    _objs[h] = o
    return h


def _get(h, cls=None):
    o = _objs.get(int(h))
    if o is None:
        raise RadiaError(f"Radia::Error002: the element {h} does not exist")
    if cls is not None and not isinstance(o, cls):
        raise RadiaError(f"Radia::Error003: element {h} has the wrong type for this function")
    return o


def _v3(x, name="vector"):
    a = np.asarray(x, dtype=np.float64).reshape(-1)
    if a.size != 3:
        raise RadiaError(f"Radia::Error000: {name} must have 3 components")
    return a


# --------------------------------------------------------------------------
# objects
# --------------------------------------------------------------------------
def ObjRecMag(P, L, M=(0.0, 0.0, 0.0)) -> int:
    """Rectangular block, centre P, dimensions L, magnetization M (radpy.cpp:3342)."""
    L = _v3(L, "dimensions")
    if np.any(L < 0):
        raise RadiaError("Radia::Error001: negative dimensions")
    return _add(RecMag(_v3(P), L, _v3(M)))


def ObjRecCur(P, L, J) -> int:
    """Current-carrying rectangular block with current density J (A/mm^2)."""
    L = _v3(L, "dimensions")
    if np.any(L < 0):
        raise RadiaError("Radia::Error001: negative dimensions")
    return _add(RecMag(_v3(P), L, np.zeros(3), _v3(J)))


def ObjPolyhdr(V, F, M=(0.0, 0.0, 0.0)) -> int:
    """Uniformly magnetized convex polyhedron; F lists 1-based vertex indices."""
    faces = [[int(i) - 1 for i in f] for f in F]
    return _add(Polyhedron(np.asarray(V, dtype=np.float64), faces, _v3(M)))


def _abs_rand_magnitude(a: float) -> float:
    """radTConvergRepair::AbsRandMagnitude (cpp/src/core/radcnvrg.h:85-91)."""
    abs_r, rel_r, zero_r = _rand
    m = max(abs_r, rel_r * a)
    return m if a != 0.0 else max(m, zero_r)


def _thckpgn_rectangle(pts: np.ndarray):
    """Centre and sides of an axis-aligned 4-point polygon, or None
    (CheckIfExtrudedPolygonIsRecMag, cpp/src/core/radappl.h:339-372).  The
    tolerance is twice the randomization magnitude, so with FldLenRndSw('off')
    no polygon qualifies."""
    if pts.shape[0] != 4:
        return None
    d1 = np.linalg.norm(pts[2] - pts[0])
    d2 = np.linalg.norm(pts[3] - pts[1])
    tol = 2.0 * _abs_rand_magnitude(max(d1, d2))
    if abs(d2 - d1) > tol:
        return None
    e = np.abs(np.roll(pts, -1, axis=0) - pts)     # |p1-p0|, |p2-p1|, |p3-p2|, |p0-p3|
    small, big = e < tol, e > tol
    alt1 = small[0, 0] and big[0, 1] and big[1, 0] and small[1, 1] and small[2, 0] and big[2, 1] and big[3, 0] and small[3, 1]
    alt2 = big[0, 0] and small[0, 1] and small[1, 0] and big[1, 1] and big[2, 0] and small[2, 1] and small[3, 0] and big[3, 1]
    if not (alt1 or alt2):
        return None
    cen, dim = np.zeros(2), np.zeros(2)
    for k in range(2):   # the longer of the first two sides along each 2-D axis
        da, db = abs(pts[1, k] - pts[0, k]), abs(pts[2, k] - pts[1, k])
        if da > db:
            cen[k], dim[k] = 0.5 * (pts[1, k] + pts[0, k]), da
        else:
            cen[k], dim[k] = 0.5 * (pts[2, k] + pts[1, k]), db
    return cen, dim


def ObjThckPgn(x, lx, pts, a="x", M=(0.0, 0.0, 0.0)) -> int:
    """Extruded convex polygon (radpy ObjThckPgn, radpy.cpp:190-225;
    radTApplication::SetExtrudedPolygon, radapl1.cpp:318-480).

    The polygon [[u, v], ...] is extruded over [x - lx/2, x + lx/2] along
    a.  As in the reference, an axis-aligned rectangle becomes a block
    (within the randomization tolerance: never with FldLenRndSw('off')); any
    other polygon is built along x in its own frame, u -> y and v -> z, and for
    a = 'y' or 'z' carries the orientation transform of
    FindSpaceTransToOrientObjAlongMainAxis (radapl1.cpp:1486-1560): a rotation
    about (1, 1, 1) by 2 pi / 3 or 4 pi / 3, with M taken back into the
    element's frame.  The extruded polygon is a polyhedron here, relaxed and
    evaluated by the polyhedron kernels (the reference's GPU assembly declines
    it, radgpu_asm.cpp:228-233)."""
    pts = np.asarray(pts, dtype=np.float64).reshape(-1, 2)
    ax = str(a)[:1].lower()
    if ax not in ("x", "y", "z"):
        raise RadiaError("Radia::Error000: ObjThckPgn: orientation definition should be 'x', 'y' or 'z'")
    if pts.shape[0] < 3:
        raise RadiaError("Radia::Error048: a face needs at least 3 points")
    M = _v3(M)
    x, lx = float(x), float(lx)
    rect = _thckpgn_rectangle(pts)
    if rect is not None:
        (cu, cv), (du, dv) = rect
        c = {"x": [x, cu, cv], "y": [cv, x, cu], "z": [cu, cv, x]}[ax]
        d = {"x": [lx, du, dv], "y": [dv, lx, du], "z": [du, dv, lx]}[ax]
        return _add(RecMag(np.array(c), np.array(d), M))
    n = pts.shape[0]
    lo, hi = x - 0.5 * lx, x + 0.5 * lx
    V = [[lo, pts[k, 0], pts[k, 1]] for k in range(n)] + [[hi, pts[k, 0], pts[k, 1]] for k in range(n)]
    F = [list(range(n)), list(range(n, 2 * n))]
    for k in range(n):
        k2 = (k + 1) % n
        F.append([k, k2, n + k2, n + k])
    if ax == "x":
        return _add(Polyhedron(np.asarray(V), F, M))
    t = trf_rotation(np.zeros(3), np.ones(3), (2.0 if ax == "y" else 4.0) * math.pi / 3.0)
    o = Polyhedron(np.asarray(V), F, (t.Minv @ M) / t.s)
    o.add_transform(1, t)
    return _add(o)


def _ccw(p: np.ndarray) -> np.ndarray:
    """The polygon counter-clockwise (signed area >= 0)."""
    x, y = p[:, 0], p[:, 1]
    area2 = float(np.dot(x, np.roll(y, -1)) - np.dot(np.roll(x, -1), y))
    return p if area2 >= 0.0 else p[::-1].copy()


def _is_convex(p: np.ndarray, tol: float) -> bool:
    """Every turn of the counter-clockwise polygon is a left turn or straight
    (radTPolygon::CheckIfConvex, called from its constructors, radplnr1.cpp:136)."""
    q = _ccw(p)
    d = np.roll(q, -1, axis=0) - q
    cr = d[:, 0] * np.roll(d, -1, axis=0)[:, 1] - d[:, 1] * np.roll(d, -1, axis=0)[:, 0]
    return bool(np.all(cr >= -tol * tol))


def _strictly_convex_crease(A: np.ndarray, B: np.ndarray, C: np.ndarray, za: float, zb: float, zc: float,
                            tol: float) -> bool:
    """Whether the two slabs A-B and B-C meet at every edge of B with a
    strictly convex crease.  The section at zb of the hull of A and C is the
    Minkowski combination t A + (1 - t) C; the crease at an edge of B is
    convex when that section lies inside the edge's line by more than tol.
    A flat crease counts as not convex, as in the reference's test
    (SetUpOnePolyhedronSegment, radapl4.cpp:716-752)."""
    t = (zc - zb) / (zc - za)
    q = _ccw(B)
    d = np.roll(q, -1, axis=0) - q
    for k in range(q.shape[0]):
        L = math.hypot(d[k, 0], d[k, 1])
        if L <= tol:
            continue
        n = np.array([d[k, 1], -d[k, 0]]) / L        # outward normal of a CCW edge
        hA, hC = float(np.max(A @ n)), float(np.max(C @ n))
        if t * hA + (1.0 - t) * hC >= float(q[k] @ n) - tol:
            return False
    return True


def _hull_faces(P: np.ndarray, tol: float) -> List[List[int]]:
    """Faces of the convex hull of the points P: hull triangles of one plane
    merged, each face's vertices ordered around it."""
    from scipy.spatial import ConvexHull

    try:
        hull = ConvexHull(P)
    except Exception as e:  # flat or degenerate set of points
        raise RadiaError(f"Radia::Error063: the slices do not enclose a volume ({e.__class__.__name__})")
    # neighbouring triangles of one plane belong to one face (union-find over
    # the hull's triangle adjacency: linear in the number of triangles)
    eqs = hull.equations
    root = list(range(len(eqs)))

    def find(i):
        while root[i] != i:
            root[i] = root[root[i]]
            i = root[i]
        return i

    for i, nb in enumerate(hull.neighbors):
        for j in nb:
            j = int(j)
            if j > i and float(np.dot(eqs[i, :3], eqs[j, :3])) > 1.0 - 1e-12 and abs(eqs[i, 3] - eqs[j, 3]) <= tol:
                root[find(j)] = find(i)
    planes: Dict[int, List[Any]] = {}
    for i, s in enumerate(hull.simplices):
        g = planes.setdefault(find(i), [eqs[i, :3].copy(), set()])
        g[1].update(int(k) for k in s)
    faces = []
    for n, idx in planes.values():
        idx = sorted(idx)
        c = P[idx].mean(axis=0)
        u = P[idx[0]] - c
        u /= np.linalg.norm(u)
        w = np.cross(n, u)
        ang = [math.atan2(float((P[i] - c) @ w), float((P[i] - c) @ u)) for i in idx]
        faces.append([idx[k] for k in np.argsort(ang)])
    return faces


def ObjMltExtPgn(slices, M=(0.0, 0.0, 0.0)) -> int:
    """Convex polyhedra from polygon slices (radpy ObjMltExtPgn,
    radpy.cpp:358-410; radTApplication::SetMultGenExtrPolygon, radapl1.cpp:859;
    SetUpPolyhedronsFromLayerPolygons / SetUpOnePolyhedronSegment,
    radapl4.cpp:435-...; CheckLayerPolygonStructures, radapl4.cpp:1036).

    slices = [[[[x, y], ...], z], ...] with z strictly increasing or strictly
    decreasing; a slice of 3 points or more is a convex polygon, fewer points
    are allowed (a pole, an edge).  Consecutive slabs stay in one polyhedron
    while they meet with a strictly convex crease at every edge of the slice
    between them; a flat or reflex crease, a slice of fewer than 3 points
    between them, or a single-point slice above ends the polyhedron there.
    Each polyhedron is built as the convex hull of its slices, so the solid
    (and the field of a uniform M) is the reference's.  One polyhedron is
    returned as itself, several in a container (CheckIfGroupIsNeeded,
    radapl4.cpp:1069).  Lengths compare with 10 max(1e-9, relative
    randomization) times the z extent, the reference's RelAbsTol."""
    M = _v3(M)
    try:
        layers = [(np.asarray(s[0], dtype=np.float64).reshape(-1, 2), float(s[1])) for s in slices]
    except Exception:
        raise RadiaError("Radia::Error000: ObjMltExtPgn, incorrect slices / layers definition")
    ns = len(layers)
    if ns < 2:
        raise RadiaError("Radia::Error063: ObjMltExtPgn, number of slices / layers should be >= 2")
    z = np.array([zz for _, zz in layers])
    dz = np.diff(z)
    if not (np.all(dz > 0.0) or np.all(dz < 0.0)):
        raise RadiaError("Radia::Error063: the slice attitudes must strictly increase or strictly decrease")
    npt = [p.shape[0] for p, _ in layers]
    if min(npt) < 1 or max(npt) < 2:
        raise RadiaError("Radia::Error063: incorrect slices / layers definition")
    tol = 10.0 * max(1e-9, _rand[1]) * abs(z[-1] - z[0])
    for p, _ in layers:
        if p.shape[0] >= 3 and not _is_convex(p, tol):
            raise RadiaError("Radia::Error111: the slice polygons must be convex")
    for i in range(1, ns):
        if npt[i - 1] < 3 and npt[i] < 3 and not (npt[i - 1] == 2 and npt[i] == 2):
            raise RadiaError("Radia::Error063: two neighbouring slices of fewer than 3 points must both be segments")
    pieces, s = [], 0
    for i in range(1, ns):
        b = i - 1
        if b > s:   # slice b lies between two slabs of the current piece
            if npt[b] < 3 or not _strictly_convex_crease(layers[b - 1][0], layers[b][0], layers[i][0],
                                                         z[b - 1], z[b], z[i], tol):
                pieces.append((s, b))
                s = b
        if npt[i] == 1 or i == ns - 1:
            pieces.append((s, i))
            s = i
    hs = []
    for a, b in pieces:
        P = np.concatenate([np.column_stack([layers[k][0], np.full(npt[k], z[k])]) for k in range(a, b + 1)])
        faces = _hull_faces(P, tol)
        hs.append(_add(Polyhedron(P, faces, M)))
    return hs[0] if len(hs) == 1 else ObjCnt(hs)


def ObjCylMag(P, r: float, h: float, nseg: int, a: str = "z", M=(0.0, 0.0, 0.0)) -> int:
    """Cylinder as a prism on a regular nseg-gon (radpy ObjCylMag;
    radTApplication::SetCylMag, radapl1.cpp:1425-1482): vertices at angles
    2 pi k / nseg from the first one, at radius r about the axis through P
    along a, extruded over h about P; built as ObjThckPgn builds it, with the
    polygon's (u, v) in the plane (y, z), (z, x) or (x, y) for a = x, y, z."""
    P = _v3(P, "centre")
    r, h, nseg = float(r), float(h), int(nseg)
    if r <= 0.0:
        raise RadiaError("Radia::Error089: the radius must be positive")
    if h <= 0.0:
        raise RadiaError("Radia::Error012: the height must be positive")
    if nseg <= 0:
        raise RadiaError("Radia::Error090: the number of segments must be positive")
    ax = str(a)[:1].lower()
    if ax not in ("x", "y", "z"):
        raise RadiaError("Radia::Error000: ObjCylMag: orientation definition should be 'x', 'y' or 'z'")
    iu, iv, ia = {"x": (1, 2, 0), "y": (2, 0, 1), "z": (0, 1, 2)}[ax]
    ang = 2.0 * math.pi / nseg * np.arange(nseg)
    pts = np.column_stack([P[iu] + r * np.cos(ang), P[iv] + r * np.sin(ang)])
    return ObjThckPgn(P[ia], h, pts, ax, M)


def ObjArcPgnMag(P, a, pgn, phi, nseg: int, sym: str = "nosym", M=(0.0, 0.0, 0.0)) -> int:
    """Arc of polygonal cross-section (radpy ObjArcPgnMag, radpy.cpp:314-345;
    radTApplication::SetArcPolygon, radapl1.cpp:1027-1370).

    The axis runs along a through the 2-D point P ((y, z), (z, x) or (x, y)
    for a = x, y, z); the cross-section points [r, z] lie in the half-plane
    of the radial direction y, z or x, rotated about the axis by phi[0].
    The first sector is the polyhedron swept from phi[0] to
    phi[0] + (phi[1] - phi[0]) / nseg: the cross-section at both ends and one
    planar face per cross-section edge (a triangle where one end has r = 0,
    none where both have).  With nseg > 1 the sector is repeated by the
    rotation through the sector angle: 'sym' as nseg symmetry images of one
    element (their magnetizations rotate with them), 'nosym' as a container
    of nseg elements that each carry the rotation as their own transform and
    have the lab-frame magnetization M."""
    p2 = np.asarray(P, dtype=np.float64).reshape(-1)
    if p2.size != 2:
        raise RadiaError("Radia::Error000: ObjArcPgnMag, incorrect definition of initial center point")
    ax = str(a)[:1].lower()
    if ax not in ("x", "y", "z"):
        raise RadiaError("Radia::Error092: the orientation should be 'x', 'y' or 'z'")
    pts = np.asarray(pgn, dtype=np.float64).reshape(-1, 2)
    ph = np.asarray(phi, dtype=np.float64).reshape(-1)
    if pts.shape[0] < 3 or ph.size != 2:
        raise RadiaError("Radia::Error000: ObjArcPgnMag, incorrect definition of cross-section polygon or angles")
    if ph[1] <= ph[0] or ph[1] - ph[0] > 2.0 * math.pi:
        raise RadiaError("Radia::Error011: incorrect angles")
    nseg = int(nseg)
    if nseg <= 0:
        raise RadiaError("Radia::Error090: the number of segments must be positive")
    dphi = (ph[1] - ph[0]) / nseg
    if dphi <= 0.0 or dphi >= math.pi:
        raise RadiaError("Radia::Error094: the segment angle must be below pi")
    if str(sym) not in ("sym", "SYM", "nosym", "NOSYM"):
        raise RadiaError("Radia::Error093: the symmetry switch should be 'sym' or 'nosym'")
    M = _v3(M)
    cen = {"x": [0.0, p2[0], p2[1]], "y": [p2[1], 0.0, p2[0]], "z": [p2[0], p2[1], 0.0]}[ax]
    cen = np.array(cen)
    axis = np.eye(3)[{"x": 0, "y": 1, "z": 2}[ax]]
    rad0 = np.eye(3)[{"x": 1, "y": 2, "z": 0}[ax]]

    def radial(ang):   # rad0 rotated about the axis by ang (right-handed)
        return math.cos(ang) * rad0 + math.sin(ang) * np.cross(axis, rad0)

    r1, r2 = radial(ph[0]), radial(ph[0] + dphi)
    r = pts[:, 0]
    if np.any(r < 0.0) or int(np.sum(r == 0.0)) > 2:
        raise RadiaError("Radia::Error095: the cross-section must not cross the axis")
    n = pts.shape[0]
    V = [cen + pts[i, 0] * r1 + pts[i, 1] * axis for i in range(n)]
    idx2 = []
    for i in range(n):        # second base: points on the axis are shared
        if r[i] == 0.0:
            idx2.append(i)
        else:
            idx2.append(len(V))
            V.append(cen + pts[i, 0] * r2 + pts[i, 1] * axis)
    F = [list(range(n)), list(idx2)]
    for j in range(n):
        k = (j + 1) % n
        if r[j] <= 0.0 and r[k] <= 0.0:
            continue
        f = [j, k, idx2[k], idx2[j]]
        F.append([v for q, v in enumerate(f) if v not in f[:q]])
    V = np.array(V)
    if nseg == 1:
        return _add(Polyhedron(V, F, M))
    rot = trf_rotation(cen, axis, dphi)
    if str(sym).lower() == "sym":
        o = Polyhedron(V, F, M)
        o.add_transform(nseg, rot)
        return _add(o)
    hs = [_add(Polyhedron(V, F, M))]
    for k in range(1, nseg):
        t = trf_rotation(cen, axis, k * dphi)
        o = Polyhedron(V, F, (t.Minv @ M) / t.s)
        o.add_transform(1, t)
        hs.append(_add(o))
    return ObjCnt(hs)


def ObjDrwAtr(obj: int, rgb=None, thcn: float = 0.001) -> int:
    """Drawing attributes (radpy ObjDrwAtr, radpy.cpp:1422).  Nothing is
    drawn here; the colour and line thickness are kept on the object so that
    scripts which set them run unchanged."""
    o = _get(obj)
    if rgb is not None:
        o.drw_rgb = [float(c) for c in np.asarray(rgb, dtype=np.float64).reshape(-1)]
    o.drw_thcn = float(thcn)
    return int(obj)


def ObjFullMag(P, L, M, K, cnt: int, mat: int, rgb=None) -> int:
    """Block, colour, material, subdivision and container in one call, in the
    reference's order (RadObjFullMag, cpp/src/lib/radentry.cpp:1858-1885):
    ObjRecMag, ObjDrwAtr, MatApl when mat > 0, ObjDivMag by K, ObjAddToCnt
    when cnt > 0."""
    h = ObjRecMag(P, L, M)
    ObjDrwAtr(h, rgb, 0.001)
    if int(mat) > 0:
        h = MatApl(h, int(mat))
    h = ObjDivMag(h, K)
    if int(cnt) > 0:
        ObjAddToCnt(int(cnt), [h])
    return h


def ObjDegFre(obj: int) -> int:
    """Degrees of freedom of the relaxation (radpy ObjDegFre;
    radTApplication::ComputeNumberOfDegOfFreedom, radapl1.cpp:2017): 3 for a
    block with a material (radrec.h:206), 3 for every polyhedron whether or
    not it has one (radvlpgn.h:229), the sum over the members of a container
    or a subdivided block (radgroup.h:149-156), 0 for currents and
    backgrounds.  Symmetry images add nothing."""
    o = _get(obj)
    if isinstance(o, Container):
        return int(sum(ObjDegFre(m) for m in o.members))
    if isinstance(o, Polyhedron):
        return 3
    if isinstance(o, RecMag):
        return 3 if getattr(o, "mat", None) is not None else 0
    return 0


def ObjMltExtRtg(layers, M=(0.0, 0.0, 0.0)) -> int:
    """Convex polyhedra from rectangular slices (radpy ObjMltExtRtg,
    radpy.cpp:428; radTApplication::SetMultGenExtrRectangle, radapl1.cpp:885;
    SetUpPolyhedronsFromLayerRectangles, radapl4.cpp:1088;
    CheckLayerRectangleStructures, radapl4.cpp:1161).

    layers = [[[x, y, z], [wx, wy]], ...]: each rectangle becomes the slice
    (x -/+ wx/2, y -/+ wy/2) at z, listed counter-clockwise from its
    (xmin, ymin) corner, and the slices are built as by ObjMltExtPgn."""
    try:
        rects = [(np.asarray(l[0], dtype=np.float64).reshape(3), np.asarray(l[1], dtype=np.float64).reshape(2))
                 for l in layers]
    except Exception:
        raise RadiaError("Radia::Error000: ObjMltExtRtg, incorrect rectangle definition")
    if len(rects) < 2:
        raise RadiaError("Radia::Error063: ObjMltExtRtg, number of slices / layers should be >= 2")
    slices = []
    for c, w in rects:
        if w[0] <= 0.0 and w[1] <= 0.0:
            raise RadiaError("Radia::Error064: Incorrect input: Rectangle dimensions should be positive.")
        x0, x1, y0, y1 = c[0] - 0.5 * w[0], c[0] + 0.5 * w[0], c[1] - 0.5 * w[1], c[1] + 0.5 * w[1]
        slices.append([[[x0, y0], [x1, y0], [x1, y1], [x0, y1]], float(c[2])])
    return ObjMltExtPgn(slices, M)


def _axis_trf(P, orient: str) -> Optional[Trf]:
    """radTApplication::FindSpaceTransToOrientObjAlongMainAxis for the
    default axis 'z' (radapl1.cpp:1486-1560)."""
    o = orient.upper()
    if o == "Z":
        return None
    if o == "X":
        return trf_rotation(P, [1, 1, 1], 2.0 * math.pi / 3.0)
    if o == "Y":
        return trf_rotation(P, [1, 1, 1], 4.0 * math.pi / 3.0)
    raise RadiaError("Radia::Error000: orientation must be 'x', 'y' or 'z'")


def ObjArcCur(P, R, Phi, h, nseg, j, man_auto="man", a="z") -> int:
    """Arc current (radTApplication::SetArcCur, radapl1.cpp:1664-1712)."""
    R = list(R)
    Phi = list(Phi)
    if len(R) != 2 or R[0] < 0 or R[1] < 0 or R[1] < R[0]:
        raise RadiaError("Radia::Error010: bad radii")
    if len(Phi) != 2 or Phi[1] < Phi[0] or (Phi[1] - Phi[0]) > 2 * math.pi:
        raise RadiaError("Radia::Error011: bad angles")
    if h <= 0:
        raise RadiaError("Radia::Error012: height must be positive")
    if str(man_auto).lower() != "man":
        raise RadiaError("ObjArcCur: only the 'man' (fixed nseg) field integration is supported")
    o = ArcCur(_v3(P), R[0], R[1], Phi[0], Phi[1], h, j, max(int(nseg), 1))
    t = _axis_trf(_v3(P), a)
    if t is not None:
        o.add_transform(1, t)
    return _add(o)


def ObjRaceTrk(P, R, L, h, nseg, j, man_auto="man", a="z") -> int:
    """Racetrack = 4 arcs + straight current blocks (radapl1.cpp:1879-1975)."""
    P = _v3(P)
    R = list(R)
    L = list(L)
    if len(R) != 2 or R[0] < 0 or R[1] < 0 or R[1] < R[0]:
        raise RadiaError("Radia::Error010: bad radii")
    if len(L) != 2 or L[0] < 0 or L[1] < 0:
        raise RadiaError("Radia::Error029: bad straight section lengths")
    if h <= 0:
        raise RadiaError("Radia::Error012: height must be positive")
    pi = 3.14159265358979324
    arcs = []
    for cx, cy, p0, p1 in ((+1, +1, 0.0, 0.5 * pi), (-1, +1, 0.5 * pi, pi),
                           (-1, -1, pi, 1.5 * pi), (+1, -1, 1.5 * pi, 1.999999999999 * pi)):
        arcs.append(ObjArcCur([P[0] + cx * 0.5 * L[0], P[1] + cy * 0.5 * L[1], P[2]], R, [p0, p1],
                              h, nseg, j, man_auto, "z"))
    members = list(arcs)
    if L[1] != 0.0:
        er = 0.5 * (L[0] + R[0] + R[1])
        d = [R[1] - R[0], L[1], h]
        members.append(ObjRecCur([P[0] + er, P[1], P[2]], d, [0.0, j, 0.0]))
        members.append(ObjRecCur([P[0] - er, P[1], P[2]], d, [0.0, -j, 0.0]))
    if L[0] != 0.0:
        er = 0.5 * (L[1] + R[0] + R[1])
        d = [L[0], R[1] - R[0], h]
        members.append(ObjRecCur([P[0], P[1] + er, P[2]], d, [-j, 0.0, 0.0]))
        members.append(ObjRecCur([P[0], P[1] - er, P[2]], d, [j, 0.0, 0.0]))
    g = ObjCnt(members)
    t = _axis_trf(P, a)
    if t is not None:
        _get(g).add_transform(1, t)
    return g


def ObjBckg(B) -> int:
    return _add(Bckg(_v3(B)))


def ObjCnt(objs: Sequence[int]) -> int:
    for h in objs:
        _get(h)
    return _add(Container(objs))


def ObjAddToCnt(cnt: int, objs: Sequence[int]) -> int:
    c = _get(cnt, Container)
    for h in objs:
        _get(h)
    c.members = sorted(set(c.members) | set(int(h) for h in objs))
    return cnt


def ObjCntStuf(obj: int) -> List[int]:
    o = _get(obj)
    return list(o.members) if isinstance(o, Container) else [obj]


def ObjCntSize(obj: int) -> int:
    """Number of direct members of a container or a subdivided block, 0 for
    any other object (radpy ObjCntSize: the size of the radTGroup)."""
    o = _get(obj)
    return len(o.members) if isinstance(o, Container) else 0


def ObjDivMag(obj: int, k, *args, **kw) -> int:
    """Subdivide a cuboid (or every cuboid of a container) by parallel planes
    (radTRecMag::SubdivideItself, radrec.cpp:971-1082).  k = [kx,ky,kz] or
    [[kx,qx],[ky,qy],[kz,qz]] with q the last-to-first size ratio."""
    if args and isinstance(args[0], str) and args[0].lower() not in ("pln",):
        raise RadiaError("ObjDivMag: only the default parallel-plane subdivision is supported")
    kk = []
    for x in k:
        if isinstance(x, (list, tuple)):
            kk.append((float(x[0]), float(x[1]) if len(x) > 1 else 1.0))
        else:
            kk.append((float(x), 1.0))
    if len(kk) != 3:
        raise RadiaError("Radia::Error000: subdivision needs 3 numbers")
    _divide(obj, kk)
    return obj


def _divide(h: int, kk):
    o = _get(h)
    if isinstance(o, Container):
        for m in list(o.members):
            _divide(m, kk)
        return
    if not isinstance(o, RecMag) or np.any(o.j != 0.0):
        return
    (kx, qx), (ky, qy), (kz, qz) = kk
    if abs(kx - 1) < 1e-10 and abs(ky - 1) < 1e-10 and abs(kz - 1) < 1e-10:
        return
    tol = 5e-12
    q0 = []
    a1 = []
    for kq, dim in zip(kk, o.d):
        kv, qv = kq
        q0v = qv ** (1.0 / (kv - 1.0)) if abs(kv - 1.0) > tol else qv
        buf = qv * q0v - 1.0
        a1.append(dim * (q0v - 1.0) / buf if abs(buf) > tol else dim / kv)
        q0.append(q0v)
    init_dims = np.array(a1)
    init_c = o.c - 0.5 * (o.d - init_dims)
    members = []
    dims = init_dims.copy()
    c = init_c.copy()
    for ix in range(int(kx)):
        for iy in range(int(ky)):
            for iz in range(int(kz)):
                sub = RecMag(c.copy(), dims.copy(), o.m.copy())
                sub.mat = o.mat
                members.append(_add(sub))
                c[2] += 0.5 * dims[2]
                dims[2] *= q0[2]
                c[2] += 0.5 * dims[2]
            c[1] += 0.5 * dims[1]
            dims[1] *= q0[1]
            c[1] += 0.5 * dims[1]
            c[2] = init_c[2]
            dims[2] = init_dims[2]
        c[0] += 0.5 * dims[0]
        dims[0] *= q0[0]
        c[0] += 0.5 * dims[0]
        c[1] = init_c[1]
        dims[1] = init_dims[1]
    cnt = Container(members)
    cnt.trfs = list(o.trfs)
    cnt.mat = o.mat
    _objs[h] = cnt


def _objm(h: int, outer: Trf) -> list:
    o = _get(h)
    out = []
    for T in images_of(o.trfs):
        Tt = outer @ T
        if isinstance(o, Container):
            for m in o.members:
                out.extend(_objm(m, Tt))
        elif isinstance(o, (ArcCur, Bckg)) or (isinstance(o, RecMag) and np.any(o.j != 0.0)):
            continue   # current sources and backgrounds carry no magnetization
        else:
            c = o.c if isinstance(o, RecMag) else getattr(o, "centre", np.zeros(3))
            m = getattr(o, "m", np.zeros(3))
            out.append([list(map(float, Tt.point(c))), list(map(float, Tt.s * (Tt.M @ m)))])
    return out


def ObjM(obj: int):
    """Centre point(s) and magnetization(s) in the lab frame, one entry per
    member and symmetry image (radpy ObjM)."""
    o = _get(obj)
    res = _objm(int(obj), Trf.identity())
    if not isinstance(o, Container) and len(res) == 1:
        return res[0]
    return res


def ObjSetM(obj: int, M) -> int:
    o = _get(obj)
    if isinstance(o, Container):
        for m in o.members:
            ObjSetM(m, M)
    elif hasattr(o, "m"):
        o.m = _v3(M).copy()
    return obj


# --------------------------------------------------------------------------
# transformations
# --------------------------------------------------------------------------
def TrfTrsl(V) -> int:
    return _add(trf_translation(_v3(V)))


def TrfRot(P, V, phi) -> int:
    return _add(trf_rotation(_v3(P), _v3(V), float(phi)))


def TrfPlSym(P, N) -> int:
    return _add(trf_plane_sym(_v3(P), _v3(N), 1.0))


def TrfInv() -> int:
    return _add(trf_field_inversion())


def TrfCmbL(orig: int, trf: int) -> int:
    t0, t1 = _get(orig, Trf), _get(trf, Trf)
    _objs[int(orig)] = t1 @ t0
    return orig


def TrfCmbR(orig: int, trf: int) -> int:
    t0, t1 = _get(orig, Trf), _get(trf, Trf)
    _objs[int(orig)] = t0 @ t1
    return orig


def TrfMlt(obj: int, trf: int, mlt: int) -> int:
    o = _get(obj, Obj)
    o.add_transform(int(mlt), _get(trf, Trf))
    return obj


def TrfOrnt(obj: int, trf: int) -> int:
    return TrfMlt(obj, trf, 1)


def TrfZerPara(obj: int, P, N) -> int:
    """RadTrfZerPara, cpp/src/lib/radentry.cpp:1802-1822: PlSym * Inv, mult 2."""
    t = trf_field_inversion() @ trf_plane_sym(_v3(P), _v3(N), 1.0)
    _get(obj, Obj).add_transform(2, t)
    return obj


def TrfZerPerp(obj: int, P, N) -> int:
    """RadTrfZerPerp, cpp/src/lib/radentry.cpp:1825-1840: PlSym, mult 2."""
    _get(obj, Obj).add_transform(2, trf_plane_sym(_v3(P), _v3(N), 1.0))
    return obj


# --------------------------------------------------------------------------
# materials
# --------------------------------------------------------------------------
def MatLin(ksi, mr) -> int:
    """Linear anisotropic material (radTApplication::SetLinearMaterial,
    radapl2.cpp:46-84): MatLin([ksipar,ksiper], mr|[mrx,mry,mrz])."""
    ksi = list(ksi)
    if len(ksi) != 2:
        raise RadiaError("Radia::Error022: MatLin needs [ksipar, ksiper]")
    if isinstance(mr, (list, tuple, np.ndarray)):
        mrv = _v3(mr)
        if not np.any(mrv != 0.0) and ksi[0] != ksi[1]:
            raise RadiaError("Radia::Error023: zero remanence with anisotropic susceptibility")
        return _add(Material(0, (float(ksi[0]), float(ksi[1])), mr=mrv))
    return _add(Material(0, (float(ksi[0]), float(ksi[1])), mr_abs=float(mr)))


def MatSatIsoFrm(*pairs) -> int:
    """M = sum ms_i tanh(ksi_i H / ms_i); arguments [ksi_i, ms_i] (radpy.cpp:1972-2010)."""
    if not 1 <= len(pairs) <= 3:
        raise RadiaError("Radia::Error024: 1 to 3 [ksi, ms] pairs")
    ks = tuple(float(p[0]) for p in pairs)
    ms = tuple(float(p[1]) for p in pairs)
    return _add(Material(1, ks, ms, mr=np.zeros(3)))


def MatApl(obj: int, mat: int) -> int:
    m = _get(mat, Material)
    _apply_mat(int(obj), m)
    return obj


def _apply_mat(h: int, m: Material):
    o = _get(h)
    if isinstance(o, Container):
        o.mat = m
        for c in o.members:
            _apply_mat(c, m)
    elif isinstance(o, (RecMag, Polyhedron)):
        if isinstance(o, RecMag) and np.any(o.j != 0.0):
            return
        if m.kind == 0 and m.mr is None:
            m.resolve(o.m)   # raises Error107 for a zero magnetization
        o.mat = m


# --------------------------------------------------------------------------
# relaxation
# --------------------------------------------------------------------------
class Interaction:
    """Result of RlxPre: the device-resident interaction and its elements."""

    def __init__(self, pack: InteractionPack, native: "_native.NativeInteraction"):
        self.pack = pack
        self.native = native
        self.M: Optional[np.ndarray] = None
        self.H: Optional[np.ndarray] = None
        self.last_status = None

    def writeback(self, M: np.ndarray):
        for e, lf in enumerate(self.pack.leaves):
            lf.obj.m = M[3 * e:3 * e + 3].copy()
        self.M = M


# RlxPre storage / solver selection; new method numbers are listed in
# RlxAuto's docstring.
_STORE = {"f32": 0, "f64": 1, "mixed": 2}


def RlxPre(obj: int, srcobj: int = 0, use_gpu=True, storage: str = "f32", fast: bool = False) -> int:
    """Builds the interaction for obj (and the extra source srcobj) on the
    device.  storage='f32' keeps the reference's FP32 matrix; 'f64' an FP64
    matrix; 'mixed' both (FP32 for the tensor-core factorization, FP64 for
    the refinement residual).  fast=True assembles polyhedron blocks with the
    vertex/edge form instead of the reference's face-by-face form."""
    pack = pack_interaction(_objs, int(obj), int(srcobj), tuple(_rand))
    nat = _native.NativeInteraction(pack, _STORE[storage] | (16 if fast else 0))
    _last_asm[0] = "gpu"
    return _add(Interaction(pack, nat))


def _status_list(st):
    return [float(st[0]), float(st[1]), float(st[2]), int(st[3])]


def RlxAuto(intrc: int, prec: float, maxiter: int, meth: int = 4, *opts) -> list:
    """Automatic relaxation (radpy RlxAuto).  meth 3/4/5/8/9/10 run the
    device-resident Jacobi/Anderson solver (same fixed point as the
    reference's methods), 11 the Newton-Krylov solver.  New: 12 = dense FP64
    LU direct solve, 13 = FP32 LU with tensor-core updates (FP16 or TF32
    operands) + FP64 GMRES refinement (linear materials only).  Options 'ZeroM->True|False', 'omega->x'.
    Returns [misfit, max|M|, max|H|, iterations]."""
    it = _get(intrc, Interaction)
    reset, omega = True, 0.0
    for o in opts:
        if not isinstance(o, str) or "->" not in o:
            continue
        key, val = [s.strip() for s in o.split("->", 1)]
        if key.lower() == "zerom":
            reset = val.lower() in ("true", "1", "yes")
        elif key.lower() == "omega":
            omega = float(val)
    n = it.pack.elem_src.shape[0]
    M0 = np.zeros(3 * n)
    if not reset:
        for e, lf in enumerate(it.pack.leaves):
            M0[3 * e:3 * e + 3] = lf.obj.m
    if meth in (12, 13):
        if np.any(it.pack.mat_kind != 0):
            raise RadiaError("RlxAuto: direct solve (meth 12/13) needs linear materials")
        M, st = it.native.direct(0 if meth == 12 else 1, min(prec, 1e-12) if meth == 12 else 1e-13, maxiter)
        st = [st[0], float(np.max(np.linalg.norm(M.reshape(-1, 3), axis=1))), 0.0, st[1]]
    else:
        method = 1 if meth == 11 else 0
        M, H, st = it.native.relax(method, prec, maxiter, reset, omega, M0)
        it.H = H
    it.writeback(M)
    it.last_status = st
    return _status_list(st)


def Solve(obj: int, prec: float, maxiter: int, meth: int = 4, *opts) -> list:
    """RlxPre + RlxAuto (radapl2.cpp:1521-1601)."""
    storage = "f64" if meth == 12 else "f32"
    h = RlxPre(obj, storage=storage)
    try:
        return RlxAuto(h, prec, maxiter, meth, *opts)
    finally:
        UtiDel(h)


# --------------------------------------------------------------------------
# field
# --------------------------------------------------------------------------
_COMP = {"b": (0, None), "h": (1, None), "m": (2, None)}


def _parse_id(fid: str):
    s = fid.lower()
    out = []
    i = 0
    while i < len(s):
        ch = s[i]
        if ch not in "bhm":
            raise RadiaError(f"Radia::Error000: unsupported field id '{fid}'")
        if i + 1 < len(s) and s[i + 1] in "xyz":
            out.append((ch, "xyz".index(s[i + 1])))
            i += 2
        else:
            out.append((ch, None))
            i += 1
    return out


def Fld(obj: int, fid: str, pts, use_gpu=True, precision: str = "double"):
    """Field at one point or a list of points (radpy Fld, radpy.cpp:2389-2445)."""
    parts = _parse_id(fid)
    P = np.asarray(pts, dtype=np.float64)
    single = P.ndim == 1
    P = P.reshape(-1, 3)
    geom = pack_sources(_objs, int(obj), tuple(_rand))
    # 'double': FP64, face-by-face polygon form (the reference's); 'single':
    # FP32 terms with FP64 accumulation; 'fast': FP64 vertex/edge polyhedron form
    prec = {"double": 0, "single": 1, "fast": 2}.get(str(precision).lower())
    if prec is None:
        raise RadiaError("Radia::Error000: precision must be 'double', 'single' or 'fast'")
    need = sorted({p[0] for p in parts})
    vals = {}
    for w in need:
        vals[w] = _native.field(geom, P, {"b": 0, "h": 1, "m": 2}[w], prec)
    _last_fld[0] = "gpu"
    if isinstance(pts, np.ndarray) and pts.ndim == 2:
        # array in, array out (an extension: the reference returns lists)
        cols = []
        for ch, comp in parts:
            cols.append(vals[ch] if comp is None else vals[ch][:, comp:comp + 1])
        return cols[0] if len(cols) == 1 else np.concatenate(cols, axis=1)
    res = []
    for i in range(P.shape[0]):
        row = []
        for ch, comp in parts:
            v = vals[ch][i]
            if comp is None:
                row.extend(float(x) for x in v)
            else:
                row.append(float(v[comp]))
        res.append(row[0] if len(row) == 1 else row)
    return res[0] if single else res


def FldLst(obj: int, fid: str, P1, P2, np_: int, arg: str = "noarg", strt: float = 0.0):
    P1, P2 = _v3(P1), _v3(P2)
    t = np.linspace(0.0, 1.0, int(np_))
    pts = P1[None, :] + t[:, None] * (P2 - P1)[None, :]
    vals = Fld(obj, fid, pts)
    if arg == "arg":
        step = np.linalg.norm(P2 - P1) / max(int(np_) - 1, 1)
        return [[strt + i * step, v] for i, v in enumerate(vals)]
    return vals


def _fldint_items(cmpn: str):
    """Quantities and output layout of a field-integral id string.

    Which integrals are computed follows ValidateFieldIntChar
    (cpp/src/core/radapl1.cpp:132-168); the order and count of the returned
    values follow radTSend::OutFieldIntCompRes (cpp/src/core/radsend.cpp:888-1003):
    'ibx' -> Ib.x, 'ib' / 'i' / '' -> Ib (3 values), 'ihz' -> Ih.z, a bare
    'x' / 'y' / 'z' not preceded by i, b or h -> that component of Ib."""
    s = str(cmpn)
    low = s.lower()
    i_used = "i" in low
    ib = (not s) or ("b" in low)
    ih = "h" in low
    if not ib and not ih:
        if not i_used:
            raise RadiaError("Radia::Error032: Incorrect input: Field Integral component identification string "
                             "should contain either combination of characters I,i,B,b,H,h,x,y,z or nothing.")
        ib = True
    n_items = 0
    prev = ""
    for ch in low:
        if ch in "bh" or (ch in "xyz" and prev not in ("b", "h")):
            n_items += 1
        prev = ch
    walk = low if (low and not (i_used and n_items == 0)) else "ib"
    items = []
    for k, ch in enumerate(walk):
        nxt = walk[k + 1] if k + 1 < len(walk) else ""
        prv = walk[k - 1] if k > 0 else ""
        comp = "xyz".index(nxt) if nxt and nxt in "xyz" else None
        if ch == "i":
            if comp is not None:
                items.append(("b", comp))
            elif not (nxt and nxt in "bh"):
                items.append(("b", None))
                break
        elif ch in "bh":
            items.append((ch, comp))
        elif ch in "xyz" and not (prv and prv in "ibh"):
            items.append(("b", "xyz".index(ch)))
    return ib, ih, items


def FldInt(obj: int, inf_or_fin: str, cmpn: str, P1, P2, precision: str = "double"):
    """Field integral along a straight line (radpy FldInt, radpy.cpp:2501-2531;
    radTApplication::ComputeFieldInt, radapl3.cpp:356-385), T mm.

    'fin' integrates from P1 to P2, 'inf' over the whole line through them
    (uniform background fields contribute zero to an infinite integral, as in
    the reference).  The accuracy is the absolute PrcBInt of FldCmpCrt /
    FldCmpPrc (default 1e-3 T mm).  One value is returned as a float, more
    as a list, as in the reference."""
    mode = str(inf_or_fin)
    if mode in ("inf", "Inf", "INF"):
        infinite = True
    elif mode in ("fin", "Fin", "FIN"):
        infinite = False
    else:
        raise RadiaError("Radia::Error033: Incorrect input: Integral identification string should be either "
                         " inf  or  fin .")
    ib, ih, items = _fldint_items(cmpn)
    a, b = _v3(P1, "first point defining integration line"), _v3(P2, "second point defining integration line")
    prec = {"double": 0, "single": 1, "fast": 2}.get(str(precision).lower())
    if prec is None:
        raise RadiaError("Radia::Error000: precision must be 'double', 'single' or 'fast'")
    geom = pack_sources(_objs, int(obj), tuple(_rand))
    what = (1 if ib else 0) | (2 if ih else 0)
    out, _st = _native.field_int(geom, a, b, infinite, what, prec, _prc["PrcBInt"])
    _last_fld[0] = "gpu"
    vals = []
    for q, comp in items:
        v = out[0:3] if q == "b" else out[3:6]
        vals.extend(float(x) for x in (v if comp is None else v[comp:comp + 1]))
    return vals[0] if len(vals) == 1 else vals


def FldPtcTrj(obj: int, E: float, init, lims, np_: int):
    """Relativistic electron trajectory in the field of obj (radpy FldPtcTrj,
    radpy.cpp:2537-2569; radTApplication::ComputeParticleTrajectory,
    radapl3.cpp:639-672): energy E (GeV), init [x0, dx/dy0, z0, dz/dy0] at
    y = lims[0], tabulated at np_ points to lims[1].  Returns np_ lists
    [y, x, dx/dy, z, dz/dy] (one flat list when np_ == 1).  With PrcCoord or
    PrcAngle set positive (FldCmpCrt / FldCmpPrc) every interval is
    integrated with step-doubling control, else with one fourth-order
    Runge-Kutta step, as in the reference.  An extension: init given as an
    [n, 4] array runs n trajectories at once (one CTA each) and returns an
    [n, np_, 5] array."""
    ini = np.asarray(init, dtype=np.float64)
    lim = np.asarray(lims, dtype=np.float64).reshape(-1)
    if lim.size != 2:
        raise RadiaError("Radia::Error000: FldPtcTrj, incorrect definition of Y range")
    batch = ini.ndim == 2
    if (batch and ini.shape[1] != 4) or (not batch and ini.size != 4):
        raise RadiaError("Radia::Error000: FldPtcTrj, incorrect definition of initial conditions")
    n = int(np_)
    if n < 1 or not (float(E) > 0):
        raise RadiaError("Radia::Error000: FldPtcTrj: incorrect or missing function argument")
    on = _prc["PrcCoord"] > 0 or _prc["PrcAngle"] > 0
    prec = [_prc["PrcCoord"], _prc["PrcAngle"], _prc["PrcCoord"], _prc["PrcAngle"]] if on else None
    geom = pack_sources(_objs, int(obj), tuple(_rand))
    try:
        out = _native.trajectories(geom, float(E), ini.reshape(-1, 4), lim[0], lim[1], n, prec)
    except RuntimeError as e:
        msg = str(e)
        k = msg.find("Radia::Error")
        raise RadiaError(msg[k:] if k >= 0 else msg) from None
    _last_fld[0] = "gpu"
    if batch:
        return out
    rows = [[float(v) for v in r] for r in out[0]]
    return rows[0] if n == 1 else rows


def FldCmpCrt(prcB: float, prcA: float, prcBint: float, prcFrc: float, prcTrjCrd: float, prcTrjAng: float) -> int:
    """Absolute accuracy levels (radpy FldCmpCrt, radpy.cpp:2845-2865;
    SetCompCriterium, radapl2.cpp:2056-2075).  Of these, FldInt uses prcBint."""
    vals = [float(v) for v in (prcB, prcA, prcBint, prcFrc, prcTrjCrd, prcTrjAng)]
    if any(not (v > 0) for v in vals):
        raise RadiaError("Radia::Error000: FldCmpCrt: incorrect or missing function argument")
    for k, v in zip(("PrcB", "PrcA", "PrcBInt", "PrcForce", "PrcCoord", "PrcAngle"), vals):
        _prc[k] = v
    return 1


def FldCmpPrc(opts: str) -> int:
    """Accuracy levels by option string 'PrcB->v,PrcBInt->v,...' (radpy
    FldCmpPrc, radpy.cpp:2870-2895; SetCompPrecisions, radapl2.cpp:2029-2052)."""
    text = str(opts).replace(" ", "")
    parts = [p for p in text.replace(";", ",").split(",") if p]
    upd = {}
    for p in parts:
        name, sep, val = p.partition("->")
        if not sep or name not in _PRC_DEFAULT:
            raise RadiaError("Radia::Error057: Incorrect input: Improper definition of absolute precision "
                             "value(s). See the usage message for the function.")
        try:
            upd[name] = float(val)
        except ValueError:
            raise RadiaError("Radia::Error057: Incorrect input: Improper definition of absolute precision "
                             "value(s). See the usage message for the function.") from None
    _prc.update(upd)
    return 1


def FldLenRndSw(onoff: str) -> int:
    """Switches the length randomization guards (radapl2.cpp:2096-2111).
    Unlike the reference, geometry is never jittered at creation; only the
    near-singularity guard magnitudes change."""
    s = onoff.lower()
    if s == "on":
        _rand[:] = _rand_on
        return 1
    if s == "off":
        _rand[:] = [0.0, 0.0, 0.0]
        return 0
    raise RadiaError("Radia::Error043: 'on' or 'off' expected")


def FldLenTol(absv: float = 1e-9, relv: float = 1e-11, zerov: float = 0.0) -> int:
    _rand_on[:] = [abs(absv), abs(relv), abs(zerov) if zerov else abs(absv)]
    _rand[:] = _rand_on
    return 1


# --------------------------------------------------------------------------
# utilities
# --------------------------------------------------------------------------
def UtiDel(h: int) -> int:
    o = _objs.pop(int(h), None)
    if isinstance(o, Interaction):
        o.native.free()
    return 0


def UtiDelAll() -> int:
    """Deletes every object; the device memory that freed interactions left
    for reuse goes back to the driver."""
    for h in list(_objs):
        UtiDel(h)
    _next[0] = 1
    model.clear_source_cache()
    _native.release_cached_memory()
    return 0


_DMP_MAGIC = b"RADB200DMP\x01"


def _dmp_closure(handles: Sequence[int]) -> Dict[int, Any]:
    """Every object reachable from the handles (container members)."""
    out: Dict[int, Any] = {}
    stack = [int(h) for h in handles]
    while stack:
        h = stack.pop()
        if h in out:
            continue
        o = _get(h)
        out[h] = o
        if isinstance(o, Container):
            stack.extend(o.members)
    return out


def _dmp_asc(h: int, o) -> str:
    lines = [f"Index: {h}"]
    if isinstance(o, Interaction):
        lines.append(f"   Relaxation interaction of {len(o.pack.leaves)} elements (device-resident)")
    elif isinstance(o, Container):
        lines.append(f"   Container of {len(o.members)} objects: {o.members}")
    elif isinstance(o, RecMag):
        lines.append("   Rectangular parallelepiped with " + ("current" if np.any(o.j != 0) else "magnetization"))
        lines.append(f"   {{x,y,z}}= {{{o.c[0]},{o.c[1]},{o.c[2]}}}")
        lines.append(f"   {{wx,wy,wz}}= {{{o.d[0]},{o.d[1]},{o.d[2]}}}")
        lines.append(f"   {{mx,my,mz}}= {{{o.m[0]},{o.m[1]},{o.m[2]}}}")
    elif isinstance(o, Polyhedron):
        lines.append(f"   Polyhedron: {len(o.v)} vertices, {len(o.faces)} faces")
        lines.append(f"   {{mx,my,mz}}= {{{o.m[0]},{o.m[1]},{o.m[2]}}}")
    elif isinstance(o, ArcCur):
        lines.append(f"   Arc current: centre {list(o.c)}, r {o.rmin}..{o.rmax}, phi {o.phimin}..{o.phimax}, "
                     f"h {o.h}, j {o.j}, {o.nseg} segments")
    elif isinstance(o, Bckg):
        lines.append(f"   Uniform background field source {{bx,by,bz}}= {{{o.b[0]},{o.b[1]},{o.b[2]}}}")
    elif isinstance(o, Material):
        lines.append(f"   Material (kind {o.kind})")
    elif isinstance(o, Trf):
        lines.append("   Space transformation")
    if isinstance(o, Obj) and o.trfs:
        lines.append(f"   {len(o.trfs)} transformation(s) attached")
    return "\n".join(lines)


def UtiDmp(elem, fmt: str = "asc"):
    """Dump of objects (radpy UtiDmp; the reference's dump,
    radintrc.cpp:1516, covers the object tree).  'asc': a text description.
    'bin': bytes that UtiDmpPrs turns back into objects in this or another
    process -- every object reachable from elem (containers, materials,
    transformations) and, for an interaction from RlxPre, its device state
    (matrix, external field, magnetization, LU factors) so that the solution
    state survives a restart without reassembly.  The binary form is this
    library's own (not the reference's byte layout); load only dumps you
    made, like any pickle-based format."""
    handles = [int(x) for x in (elem if isinstance(elem, (list, tuple)) else [elem])]
    f = str(fmt).lower()
    if f.startswith("asc"):
        return "\n".join(_dmp_asc(h, _get(h)) for h in handles)
    if not f.startswith("bin"):
        raise RadiaError("Radia::Error000: UtiDmp: format must be 'asc' or 'bin'")
    objs: Dict[int, Any] = {}
    intrc: Dict[int, Any] = {}
    for h in handles:
        o = _get(h)
        if isinstance(o, Interaction):
            intrc[h] = {"pack": o.pack, "storage": o.native.storage, "state": o.native.save(), "M": o.M}
        else:
            objs.update(_dmp_closure([h]))
    payload = {"roots": handles, "single": not isinstance(elem, (list, tuple)), "objs": objs, "intrc": intrc}
    return _DMP_MAGIC + pickle.dumps(payload, protocol=4)


class _DmpUnpickler(pickle.Unpickler):
    """Only this package's model classes, numpy arrays and builtins."""
    _ok_modules = ("radiacuda_b200.model", "numpy", "numpy.core.multiarray", "numpy._core.multiarray",
                   "numpy.core.numeric", "numpy._core.numeric", "builtins", "collections")

    def find_class(self, module, name):
        if module in self._ok_modules and not name.startswith("_") or (module.endswith("multiarray") and
                                                                       name == "_reconstruct"):
            if module == "builtins" and name not in ("list", "dict", "tuple", "set", "frozenset", "int", "float",
                                                     "complex", "bool", "str", "bytes", "slice", "range"):
                raise pickle.UnpicklingError(f"UtiDmpPrs: {module}.{name} not allowed")
            return super().find_class(module, name)
        raise pickle.UnpicklingError(f"UtiDmpPrs: {module}.{name} not allowed")


def UtiDmpPrs(bstr: bytes):
    """Instantiates the objects (and interactions) of a UtiDmp(..., 'bin')
    dump under new handles (radpy UtiDmpPrs); returns the new handle of the
    dumped element, or a list for a dumped list."""
    b = bytes(bstr)
    if not b.startswith(_DMP_MAGIC):
        raise RadiaError("Radia::Error000: UtiDmpPrs: not a dump made by UtiDmp(..., 'bin')")
    payload = _DmpUnpickler(io.BytesIO(b[len(_DMP_MAGIC):])).load()
    remap: Dict[int, int] = {}
    # new handles in the old handles' order: containers iterate their members
    # by handle, so the traversal order (and every result) is preserved
    for old in sorted(payload["objs"]):
        remap[int(old)] = _add(payload["objs"][old])
    for o in payload["objs"].values():
        if isinstance(o, Container):
            o.members = sorted(remap.get(m, m) for m in o.members)
    for old, rec in payload["intrc"].items():
        pack = rec["pack"]
        for lf in pack.leaves:
            lf.handle = remap.get(lf.handle, lf.handle)
        nat = _native.NativeInteraction(pack, rec["storage"], state=rec["state"])
        it = Interaction(pack, nat)
        it.M = rec["M"]
        remap[int(old)] = _add(it)
    out = [remap[int(h)] for h in payload["roots"]]
    return out[0] if payload["single"] else out


def _flat_floats(data) -> List[float]:
    """Nested lists / arrays flattened to floats, as the reference copies them
    into its share buffer (CopyPyNestedListElemsToNumAr)."""
    if isinstance(data, (list, tuple)):
        out: List[float] = []
        for d in data:
            out.extend(_flat_floats(d))
        return out
    return [float(v) for v in np.asarray(data, dtype=np.float64).reshape(-1)]


def UtiMPI(mode: str, data=None, rankFrom: int = 0, rankTo: int = -1):
    """Parallel-process control (radpy UtiMPI, radpy.cpp:3280-3335), on the
    torch.distributed default process group in place of MPI (one process
    per GPU).  'on' and 'in' return this process's rank (0 when no group is
    initialized: this library does not start one), 'off' returns it and
    leaves the group to its owner, 'barrier' waits for every rank.

    'share' follows radTApplication's MPI share (radapl1.cpp:2345-2440):
    with rankTo < 0 every rank joins a broadcast from rankFrom, whether or
    not it passes data; with rankTo >= 0 only rankFrom and rankTo take part,
    rankFrom sending the count and then the values.  A rank that passed data
    gets the shared values back, flattened to floats (its own data when it
    received nothing); a rank without data gets its rank, as in the
    reference.  rankFrom must pass data."""
    m = str(mode).strip().lower()
    if m not in ("on", "in", "off", "share", "barrier"):
        raise RadiaError("Radia::Error000: UtiMPI: the first argument should be 'on', 'in', 'off', 'share' or "
                         "'barrier'")
    dist = None
    try:
        import torch.distributed as _dist
        if _dist.is_available() and _dist.is_initialized():
            dist = _dist
    except ImportError:
        pass
    rank = dist.get_rank() if dist is not None else 0
    if m == "barrier" and dist is not None:
        dist.barrier()
    if m != "share":
        return rank
    flat = _flat_floats(data) if data is not None else None
    if dist is None:
        return rank if flat is None else flat
    src, dst = int(rankFrom), int(rankTo)
    if rank == src and flat is None:
        raise RadiaError("Radia::Error601: UtiMPI share: the sending rank has no data")
    if dst < 0:
        box = [flat if rank == src else None]
        dist.broadcast_object_list(box, src=src)
        return rank if flat is None else [float(v) for v in box[0]]
    if rank not in (src, dst):
        return rank if flat is None else flat
    import torch
    dev = (torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl"
           else torch.device("cpu"))
    if rank == src:
        dist.send(torch.tensor([len(flat)], dtype=torch.int64, device=dev), dst)
        if flat:
            dist.send(torch.tensor(flat, dtype=torch.float64, device=dev), dst)
        return flat
    cnt = torch.zeros(1, dtype=torch.int64, device=dev)
    dist.recv(cnt, src)
    buf = torch.empty(int(cnt.item()), dtype=torch.float64, device=dev)
    if buf.numel():
        dist.recv(buf, src)
    return rank if flat is None else [float(v) for v in buf.cpu().tolist()]


def UtiVer() -> float:
    return 4.32


def UtiFldLastBackend() -> str:
    return _last_fld[0]


def UtiAsmLastBackend() -> str:
    return _last_asm[0]


def UtiGpuFallback(mode: Optional[str] = None) -> str:
    """Policy when the device cannot hold the interaction.  This library has
    no CPU fallback: 'cpu' and 'break' both raise on such a failure; the
    setting is kept for API compatibility."""
    if mode is not None:
        if mode not in ("cpu", "break", "gpu_streaming"):
            raise RadiaError("Radia::Error000: mode must be 'cpu', 'break' or 'gpu_streaming'")
        _fallback[0] = mode
    return _fallback[0]
