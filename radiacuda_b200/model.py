"""Object model and packer behind the ``rad`` API.

Radia keeps magnetized volumes, coils and containers in a handle map and walks
that tree every time it assembles an interaction or evaluates a field.  This
module holds the same tree (construction is not on the hot path) and flattens
it into the plain arrays of ``include/radb200.h`` that the CUDA library
consumes:

* every leaf becomes one source record (cuboid, polyhedron, arc current,
  background) plus a contiguous run of image transforms in one transform
  table -- the symmetry / orientation images of Radia's transform lists are
  NOT duplicated into records, the kernels apply them in-kernel;
* relaxable leaves (cuboids and polyhedra with a material) become the
  elements of the interaction matrix, in Radia's traversal order
  (radTInteraction::CountMainRelaxElems, cpp/src/core/radintrc.cpp:249-345).

Transform semantics follow gmTrans (ext/genmath/gmtrans.h:22-84) and the image
enumeration of radTInteraction::NestedFor_Trans (radintrc.cpp:527-553): the
transform list of a leaf is [outermost container ... own], a transform with
multiplicity m contributes powers 0..m-1, and the first image (all powers 0,
orientation transforms applied once) is the element's main transform.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

TRF_STRIDE = 24
REC_STRIDE = 12
POLY_STRIDE = 6
FACE_STRIDE = 10
ARC_STRIDE = 10
MAT_STRIDE = 12


class RadiaError(RuntimeError):
    """Raised where the reference raises RuntimeError (pyparse.h:64-80)."""


# --------------------------------------------------------------------------
# transforms
# --------------------------------------------------------------------------
@dataclass
class Trf:
    """Space transformation P -> M P + V acting on fields as F -> s M F.

    gmTrans, ext/genmath/gmtrans.h:22-84; products as radTrans Product,
    cpp/src/core/radtrans.h:197-201."""

    M: np.ndarray
    V: np.ndarray
    s: float = 1.0
    detM: float = 1.0
    Minv: Optional[np.ndarray] = None

    def __post_init__(self):
        self.M = np.asarray(self.M, dtype=np.float64).reshape(3, 3)
        self.V = np.asarray(self.V, dtype=np.float64).reshape(3)
        if self.Minv is None:
            self.Minv = np.linalg.inv(self.M)

    @staticmethod
    def identity() -> "Trf":
        return Trf(np.eye(3), np.zeros(3), 1.0, 1.0, np.eye(3))

    def __matmul__(self, other: "Trf") -> "Trf":
        # self applied after other (radtrans.h:197-201)
        return Trf(self.M @ other.M, self.M @ other.V + self.V,
                   self.s * other.s, self.detM * other.detM,
                   other.Minv @ self.Minv)

    def point(self, p):
        return self.M @ np.asarray(p, dtype=np.float64) + self.V

    def record(self) -> np.ndarray:
        r = np.zeros(TRF_STRIDE)
        r[0:9] = self.Minv.reshape(9)
        r[9:12] = self.V
        r[12:21] = (self.s * self.M).reshape(9)
        r[21] = self.s
        r[22] = self.detM
        return r


def trf_translation(v) -> Trf:
    """radTApplication::SetTranslation (radapl1.cpp, ID 1)."""
    return Trf(np.eye(3), np.asarray(v, dtype=np.float64), 1.0, 1.0, np.eye(3))


def trf_rotation(p, axis, phi) -> Trf:
    """radTApplication::SetRotation, cpp/src/core/radapl1.cpp:2168-2208."""
    a = np.asarray(axis, dtype=np.float64)
    a = a / math.sqrt(a @ a)
    x, y, z = a
    c, s = math.cos(phi), math.sin(phi)
    omc = 1.0 - c
    M = np.array([[x * x + c * (y * y + z * z), omc * x * y - s * z, omc * x * z + s * y],
                  [omc * x * y + s * z, y * y + c * (x * x + z * z), omc * y * z - s * x],
                  [omc * x * z - s * y, omc * y * z + s * x, z * z + c * (x * x + y * y)]])
    V = (np.eye(3) - M) @ np.asarray(p, dtype=np.float64)
    return Trf(M, V, 1.0, float(np.linalg.det(M)))


def trf_plane_sym(p, n, s=1.0) -> Trf:
    """radTApplication::SetPlaneSym, cpp/src/core/radapl1.cpp:2212-2233."""
    n = np.asarray(n, dtype=np.float64)
    n = n / math.sqrt(n @ n)
    M = np.eye(3) - 2.0 * np.outer(n, n)
    V = (np.eye(3) - M) @ np.asarray(p, dtype=np.float64)
    return Trf(M, V, float(s), -1.0)


def trf_field_inversion() -> Trf:
    """radTApplication::SetFieldInversion: identity map, field sign -1."""
    return Trf(np.eye(3), np.zeros(3), -1.0, 1.0, np.eye(3))


# --------------------------------------------------------------------------
# materials
# --------------------------------------------------------------------------
@dataclass
class Material:
    kind: int                      # 0 linear, 1 tanh formula, 2 table
    ksi: Tuple[float, ...] = ()    # linear: (ksi_par, ksi_perp); tanh: ksi_i
    ms: Tuple[float, ...] = ()     # tanh: ms_i
    mr: Optional[np.ndarray] = None  # remanence vector (easy axis defined)
    mr_abs: Optional[float] = None   # scalar remanence (easy axis from the object)
    table: Optional[np.ndarray] = None  # [n,3] H, M, dM/dH

    def resolve(self, magn) -> Tuple[np.ndarray, np.ndarray]:
        """chi tensor and Mr for an element with magnetization ``magn``.

        radTLinearAnisotropMaterial::SetupKsiTensor / FinishSetup,
        cpp/src/core/radmater.h:221-242,292-303."""
        if self.kind != 0:
            return np.zeros((3, 3)), np.zeros(3)
        if self.mr is not None:
            mr = self.mr
        else:
            m = np.asarray(magn, dtype=np.float64)
            am = math.sqrt(m @ m)
            if am < 1e-10:
                raise RadiaError("Radia::Error107: easy magnetization axis undefined "
                                 "(zero magnetization of the object)")
            mr = (self.mr_abs / am) * m
        amr = math.sqrt(mr @ mr)
        with np.errstate(invalid="ignore", divide="ignore"):
            L = mr / amr
        kpar, kperp = self.ksi
        chi = kperp * np.eye(3) + (kpar - kperp) * np.outer(L, L)
        return chi, mr.copy()

    def record(self, magn) -> np.ndarray:
        if self.kind == 0 and self.mr is not None:
            # independent of the element's magnetization: computed once
            cached = getattr(self, "_rec_cache", None)
            if cached is None:
                cached = self._record(None)
                object.__setattr__(self, "_rec_cache", cached)
            return cached.copy()
        return self._record(magn)

    def _record(self, magn) -> np.ndarray:
        r = np.zeros(MAT_STRIDE)
        if self.kind == 0:
            chi, mr = self.resolve(magn)
            r[0:9] = chi.reshape(9)
            r[9:12] = mr
        elif self.kind == 1:
            n = len(self.ksi)
            r[0:n] = self.ksi
            r[3:3 + n] = self.ms
            r[6] = n
        return r


# --------------------------------------------------------------------------
# objects
# --------------------------------------------------------------------------
class Obj:
    kind = "obj"

    def __init__(self):
        self.trfs: List[Tuple[int, Trf]] = []   # front = outermost

    def add_transform(self, mult: int, t: Trf):
        # radTg3d::AddTransform pushes to the front (radg3d.h:871-875)
        self.trfs.insert(0, (int(mult), t))


class RecMag(Obj):
    """Rectangular block with uniform magnetization and/or current density
    (radTRecMag, cpp/src/core/radrec.h)."""
    kind = "rec"

    def __init__(self, c, d, m, j=(0.0, 0.0, 0.0)):
        super().__init__()
        self.c = np.asarray(c, dtype=np.float64).reshape(3)
        self.d = np.asarray(d, dtype=np.float64).reshape(3)
        self.m = np.asarray(m, dtype=np.float64).reshape(3).copy()
        self.j = np.asarray(j, dtype=np.float64).reshape(3)
        self.mat: Optional[Material] = None

    @property
    def relaxable(self):
        return self.mat is not None and not np.any(self.j != 0.0)


class Polyhedron(Obj):
    """Uniformly magnetized convex polyhedron (radTPolyhedron,
    cpp/src/core/radvlpgn.h).  Face frames follow
    radTPolyhedron::FillInTransAndFacesInLocFrames (radvlpgn.cpp:350-437)."""
    kind = "poly"

    def __init__(self, verts, faces, m):
        super().__init__()
        self.v = np.asarray(verts, dtype=np.float64).reshape(-1, 3)
        self.faces = [list(f) for f in faces]
        self.m = np.asarray(m, dtype=np.float64).reshape(3).copy()
        self.mat: Optional[Material] = None
        self._build_faces()

    @property
    def relaxable(self):
        return self.mat is not None

    def _build_faces(self):
        v = self.v
        used = sorted({i for f in self.faces for i in f})
        self.centre = v[used].mean(axis=0)
        cen = self.centre
        recs, verts2d = [], []
        span = float(np.max(np.abs(v))) if v.size else 1.0
        for f in self.faces:
            if len(f) < 3:
                raise RadiaError("Radia::Error048: a face needs at least 3 points")
            p0, p1 = v[f[0]], v[f[1]]
            n = None
            for j in range(2, len(f)):
                cand = np.cross(p1 - p0, v[f[j]] - p0)
                if np.max(np.abs(cand)) > (1e-12 * max(span, 1.0)) ** 2:
                    n = cand
                    break
            if n is None:
                raise RadiaError("Radia::Error049: degenerate face")
            order = list(f)
            # outward orientation: every vertex on the inner side
            if np.dot(n, cen - p0) > 0.0:
                n = -n
                order = order[::-1]
            n = n / math.sqrt(n @ n)
            if abs(n[2] + 1.0) > 1e-09:
                inv = 1.0 / (n[2] + 1.0)
                st1 = np.array([n[1] * n[1] * inv + n[2], -n[0] * n[1] * inv, -n[0]])
                st2 = np.array([st1[1], n[0] * n[0] * inv + n[2], -n[1]])
                st3 = np.array([-st1[2], -st2[2], n[2]])
            else:
                st1 = np.array([1.0, 0.0, 0.0])
                st2 = np.array([0.0, -1.0, 0.0])
                st3 = np.array([0.0, 0.0, -1.0])
            R = np.stack([st1, st2, st3])
            loc = v[order] @ R.T
            pts = [loc[k, :2].copy() for k in range(len(order))]
            coordz = loc[-1, 2]
            pts = _ccw_2d(pts)
            rec = np.zeros(FACE_STRIDE)
            rec[0:9] = R.reshape(9)
            rec[9] = coordz
            recs.append(rec)
            verts2d.append(np.array(pts))
        self.face_rec = np.array(recs)
        self.face_v2d = verts2d


def _ccw_2d(pts):
    """radTPolygon::CheckAndRearrangeEdgePoints, radplnr1.cpp:1361-1391."""
    n = len(pts)
    cnt = 0
    p1, p2 = pts[0], pts[1]
    v1 = p2 - p1
    p1 = p2
    for i in range(2, n + 2):
        p2 = pts[0] if i == n else (pts[i] if i != n + 1 else pts[1])
        v2 = p2 - p1
        cnt += -1 if (v1[0] * v2[1] - v2[0] * v1[1]) < -1e-13 else 1
        p1, v1 = p2, v2
    if cnt < 0:
        pts = [pts[0]] + [pts[n - i] for i in range(1, n)]
    return pts


class ArcCur(Obj):
    """Current-carrying arc of rectangular cross-section (radTArcCur,
    cpp/src/core/radarccu.h:42-59), field by trapezoid integration in phi."""
    kind = "arc"

    def __init__(self, c, rmin, rmax, phimin, phimax, h, j, nseg):
        super().__init__()
        self.c = np.asarray(c, dtype=np.float64).reshape(3)
        self.rmin, self.rmax = float(rmin), float(rmax)
        self.phimin, self.phimax = float(phimin), float(phimax)
        self.h, self.j, self.nseg = float(h), float(j), int(nseg)

    relaxable = False


class Bckg(Obj):
    """Uniform background field (radTBackgroundFieldSource)."""
    kind = "bkg"

    def __init__(self, b):
        super().__init__()
        self.b = np.asarray(b, dtype=np.float64).reshape(3)

    relaxable = False


class Container(Obj):
    """radTGroup: members iterated in handle order (GroupMapOfHandlers is a
    std::map keyed by element handle)."""
    kind = "cnt"

    def __init__(self, members: Sequence[int]):
        super().__init__()
        self.members: List[int] = sorted(set(int(m) for m in members))

    relaxable = False


# --------------------------------------------------------------------------
# flattening
# --------------------------------------------------------------------------
@dataclass(slots=True)
class Leaf:
    handle: int
    obj: Obj
    trf_list: List[Tuple[int, Trf]]


def collect_leaves(objs: Dict[int, Obj], handle: int,
                   outer: Optional[List[Tuple[int, Trf]]] = None,
                   out: Optional[List[Leaf]] = None) -> List[Leaf]:
    """Depth-first walk in Radia's order (radintrc.cpp:249-345).  Leaves
    without transformations of their own share their container's list (the
    lists are only read)."""
    if outer is None:
        outer = []
    if out is None:
        out = []
    get = objs.get
    append = out.append

    def walk(h: int, outer_l: List[Tuple[int, Trf]]) -> None:
        o = get(h)
        if o is None:
            raise RadiaError(f"Radia::Error002: unknown element {h}")
        lst = outer_l + o.trfs if o.trfs else outer_l
        if not isinstance(o, Container):
            append(Leaf(h, o, lst))
            return
        for m in o.members:
            c = get(m)
            if c is not None and not c.trfs and not isinstance(c, Container):
                append(Leaf(m, c, lst))
            else:
                walk(m, lst)

    walk(handle, outer)
    return out


def images_of(trf_list: List[Tuple[int, Trf]]) -> List[Trf]:
    """All images T1^k1 T2^k2 ... (radintrc.cpp:527-553); first = main."""
    res: List[Trf] = []

    def rec(base: Trf, i: int):
        if i == len(trf_list):
            res.append(base)
            return
        mult, t = trf_list[i]
        if mult == 1:
            rec(base @ t, i + 1)
            return
        rec(base, i + 1)
        cur = base
        for _ in range(1, mult):
            cur = cur @ t
            rec(cur, i + 1)

    rec(Trf.identity(), 0)
    return res


class Packed:
    """numpy arrays matching RadB200Geom (and RadB200Relax)."""

    def __init__(self):
        self.trf: List[np.ndarray] = []
        self.rec: List[np.ndarray] = []
        self.rec_img: List[Tuple[int, int]] = []
        self.rec_handles: List[int] = []
        self.poly: List[np.ndarray] = []
        self.poly_info: List[Tuple[int, int, int, int]] = []
        self.poly_handles: List[int] = []
        self.face: List[np.ndarray] = []
        self.face_vtx: List[Tuple[int, int]] = []
        self.vtx: List[np.ndarray] = []
        self.n_vtx = 0
        self.arc: List[np.ndarray] = []
        self.arc_img: List[Tuple[int, int]] = []
        self.bkg: List[np.ndarray] = []
        self.bkg_img: List[Tuple[int, int]] = []
        self.abs_rand = self.rel_rand = self.zero_rand = 0.0
        # leaves with the same transform chain (the same Trf objects, e.g. all
        # the untransformed members of a mesh) share one run of image records
        self._chains: Dict[tuple, Tuple[int, int, List["Trf"]]] = {}
        self.last_images: List["Trf"] = []

    def _images(self, trf_list) -> Tuple[int, int]:
        key = tuple((mult, id(t)) for mult, t in trf_list)
        hit = self._chains.get(key)
        if hit is None:
            ims = images_of(trf_list)
            first = len(self.trf)
            for t in ims:
                self.trf.append(t.record())
            hit = (first, len(ims), ims)
            self._chains[key] = hit
        self.last_images = hit[2]
        return hit[0], hit[1]

    def add_leaf(self, leaf: Leaf, magn=None) -> Tuple[int, int]:
        """Returns (source kind, index) with kind 0 rec, 1 poly, 2 arc, 3 bkg."""
        o = leaf.obj
        first, cnt = self._images(leaf.trf_list)
        m = o.m if magn is None and hasattr(o, "m") else magn
        if isinstance(o, RecMag):
            r = np.zeros(REC_STRIDE)
            r[0:3], r[3:6], r[6:9], r[9:12] = o.c, o.d, m, o.j
            self.rec.append(r)
            self.rec_img.append((first, cnt))
            self.rec_handles.append(leaf.handle)
            return 0, len(self.rec) - 1
        if isinstance(o, Polyhedron):
            r = np.zeros(POLY_STRIDE)
            r[0:3], r[3:6] = o.centre, m
            f0 = len(self.face)
            for k in range(o.face_rec.shape[0]):
                self.face.append(o.face_rec[k])
                v2 = o.face_v2d[k]
                self.face_vtx.append((self.n_vtx, v2.shape[0]))
                self.vtx.append(v2)
                self.n_vtx += v2.shape[0]
            self.poly.append(r)
            self.poly_info.append((f0, o.face_rec.shape[0], first, cnt))
            self.poly_handles.append(leaf.handle)
            return 1, len(self.poly) - 1
        if isinstance(o, ArcCur):
            r = np.array([o.c[0], o.c[1], o.c[2], o.rmin, o.rmax, o.phimin, o.phimax,
                          o.h, o.j, float(o.nseg)])
            self.arc.append(r)
            self.arc_img.append((first, cnt))
            return 2, len(self.arc) - 1
        if isinstance(o, Bckg):
            self.bkg.append(o.b.copy())
            self.bkg_img.append((first, cnt))
            return 3, len(self.bkg) - 1
        raise RadiaError(f"unsupported object kind {o.kind}")

    def arrays(self) -> Dict[str, np.ndarray]:
        def f64(lst, stride):
            return (np.ascontiguousarray(np.array(lst, dtype=np.float64).reshape(-1, stride))
                    if lst else np.zeros((0, stride)))

        def i32(lst, stride):
            return (np.ascontiguousarray(np.array(lst, dtype=np.int32).reshape(-1, stride))
                    if lst else np.zeros((0, stride), dtype=np.int32))

        return dict(
            trf=f64(self.trf, TRF_STRIDE),
            rec=f64(self.rec, REC_STRIDE), rec_img=i32(self.rec_img, 2),
            poly=f64(self.poly, POLY_STRIDE), poly_info=i32(self.poly_info, 4),
            face=f64(self.face, FACE_STRIDE), face_vtx=i32(self.face_vtx, 2),
            vtx2d=(np.ascontiguousarray(np.concatenate(self.vtx, axis=0)) if self.vtx
                   else np.zeros((0, 2))),
            arc=f64(self.arc, ARC_STRIDE), arc_img=i32(self.arc_img, 2),
            bkg=f64(self.bkg, 3), bkg_img=i32(self.bkg_img, 2),
            rand=np.array([self.abs_rand, self.rel_rand, self.zero_rand]),
        )


@dataclass
class InteractionPack:
    """Everything RlxPre needs: relaxable elements, their materials, and the
    external (non-relaxable) sources."""
    elems: Dict[str, np.ndarray]
    ext: Optional[Dict[str, np.ndarray]]
    elem_src: np.ndarray
    mat_kind: np.ndarray
    mat: np.ndarray
    mh: np.ndarray
    leaves: List[Leaf]
    main: List[Trf] = field(default_factory=list)


# Packed sources of recent (handle, rand) pairs.  Objects are immutable
# through the API except for their magnetization (relaxation write-back,
# ObjSetM), and transformations are only ever added; so an entry stays valid
# while the walk meets the same objects with transformation lists of the same
# lengths, and only the M columns are refreshed.  The entry holds the leaves, so no
# object id it compares can be reused while it lives.
_SRC_CACHE: Dict[Tuple[int, Tuple[float, ...]], tuple] = {}
_SRC_CACHE_MAX = 4


def _leaf_key(leaves: List[Leaf]) -> np.ndarray:
    # object identity and the length of its transformation list (transforms
    # are only ever added, at the front)
    k = np.empty((len(leaves), 2), dtype=np.int64)
    k[:, 0] = np.fromiter((id(lf.obj) for lf in leaves), dtype=np.int64, count=len(leaves))
    k[:, 1] = np.fromiter((len(lf.trf_list) for lf in leaves), dtype=np.int64, count=len(leaves))
    return k


def clear_source_cache():
    _SRC_CACHE.clear()
    _INT_CACHE.clear()


def pack_sources(objs, handle, rand) -> Dict[str, np.ndarray]:
    """Flat source arrays of the object tree under handle (RadB200Geom).
    Returns fresh arrays: callers may modify them."""
    leaves = collect_leaves(objs, handle)
    key = (int(handle), tuple(float(x) for x in rand))
    fp = _leaf_key(leaves)
    hit = _SRC_CACHE.get(key)
    if hit is not None and hit[0].shape == fp.shape and np.array_equal(hit[0], fp):
        _, arrays, slots, _ = hit
        for name, col, rows, objs_m in slots:
            if rows.size:
                arrays[name][rows, col:col + 3] = np.array([o.m for o in objs_m], dtype=np.float64)
        return {k: v.copy() for k, v in arrays.items()}
    p = Packed()
    p.abs_rand, p.rel_rand, p.zero_rand = rand
    rec_rows, rec_objs, poly_rows, poly_objs = [], [], [], []
    for lf in leaves:
        kind, idx = p.add_leaf(lf)
        if kind == 0 and hasattr(lf.obj, "m"):
            rec_rows.append(idx)
            rec_objs.append(lf.obj)
        elif kind == 1:
            poly_rows.append(idx)
            poly_objs.append(lf.obj)
    arrays = p.arrays()
    slots = [("rec", 6, np.array(rec_rows, dtype=np.int64), rec_objs),
             ("poly", 3, np.array(poly_rows, dtype=np.int64), poly_objs)]
    if len(_SRC_CACHE) >= _SRC_CACHE_MAX:
        _SRC_CACHE.pop(next(iter(_SRC_CACHE)))
    _SRC_CACHE[key] = (fp, arrays, slots, leaves)
    return {k: v.copy() for k, v in arrays.items()}


_INT_CACHE: Dict[tuple, tuple] = {}


def _int_key(leaves: List[Leaf]) -> np.ndarray:
    k = np.empty((len(leaves), 3), dtype=np.int64)
    k[:, :2] = _leaf_key(leaves)
    k[:, 2] = np.fromiter((id(getattr(lf.obj, "mat", None)) for lf in leaves), dtype=np.int64, count=len(leaves))
    return k


def _refresh_m(arrays, slots):
    for name, col, rows, objs_m in slots:
        if rows.size:
            arrays[name][rows, col:col + 3] = np.array([o.m for o in objs_m], dtype=np.float64)


def _m_slots(kinds_objs):
    rec_rows, rec_objs, poly_rows, poly_objs = [], [], [], []
    for (kind, idx), o in kinds_objs:
        if kind == 0 and hasattr(o, "m"):
            rec_rows.append(idx)
            rec_objs.append(o)
        elif kind == 1:
            poly_rows.append(idx)
            poly_objs.append(o)
    return [("rec", 6, np.array(rec_rows, dtype=np.int64), rec_objs),
            ("poly", 3, np.array(poly_rows, dtype=np.int64), poly_objs)]


def _mat_groups(relax_leaves):
    """Element rows of each material object, with the elements' objects."""
    groups: Dict[int, tuple] = {}
    for e, lf in enumerate(relax_leaves):
        mat = lf.obj.mat
        g = groups.get(id(mat))
        if g is None:
            g = groups[id(mat)] = (mat, [], [])
        g[1].append(e)
        g[2].append(lf.obj)
    return [(mat, np.array(rows, dtype=np.int64), objs_g) for mat, rows, objs_g in groups.values()]


def pack_interaction(objs, handle, srcobj, rand) -> InteractionPack:
    """Relaxable elements, their materials and the external sources of the
    object tree under handle (plus srcobj).  Cached like pack_sources: the
    entry is reused while the walk meets the same objects, transformation
    list lengths and materials; magnetizations and the material records that
    depend on them are refreshed."""
    leaves = collect_leaves(objs, handle)
    sleaves = collect_leaves(objs, srcobj) if srcobj else []
    key = (int(handle), int(srcobj), tuple(float(x) for x in rand))
    fp = _int_key(leaves + sleaves)
    hit = _INT_CACHE.get(key)
    if hit is not None and hit[0].shape == fp.shape and np.array_equal(hit[0], fp):
        _, pack, eslots, xslots, _, mgroups = hit
        _refresh_m(pack.elems, eslots)
        if pack.ext is not None:
            _refresh_m(pack.ext, xslots)
        mats = pack.mat
        for mat, rows, objs_g in mgroups:
            if mat.kind == 2:
                continue
            if mat.kind == 0 and mat.mr is not None:  # one record for all its elements
                mats[rows] = mat.record(None)
            else:
                for e, o in zip(rows, objs_g):
                    mats[e] = mat.record(o.m)
        return InteractionPack(
            elems={k: v.copy() for k, v in pack.elems.items()},
            ext=({k: v.copy() for k, v in pack.ext.items()} if pack.ext is not None else None),
            elem_src=pack.elem_src.copy(), mat_kind=pack.mat_kind.copy(), mat=mats.copy(), mh=pack.mh.copy(),
            leaves=list(pack.leaves), main=list(pack.main))
    pe, px = Packed(), Packed()
    pe.abs_rand, pe.rel_rand, pe.zero_rand = rand
    px.abs_rand, px.rel_rand, px.zero_rand = rand
    elem_src, mat_kind, mats, mh_rows, relax_leaves, mains = [], [], [], [], [], []
    eko, xko = [], []
    n_ext = 0
    for lf in leaves:
        o = lf.obj
        if getattr(o, "relaxable", False):
            kind, idx = pe.add_leaf(lf)
            eko.append(((kind, idx), o))
            elem_src.append((kind, idx))
            mat = o.mat
            rec = mat.record(o.m)
            # the main image of this element: first image of its chain
            if mat.kind == 2:
                rec[0] = len(mh_rows)
                rec[1] = mat.table.shape[0]
                mh_rows.extend(list(mat.table))
            mat_kind.append(mat.kind)
            mats.append(rec)
            relax_leaves.append(lf)
            mains.append(pe.last_images[0])
        else:
            xko.append((px.add_leaf(lf), o))
            n_ext += 1
    for lf in sleaves:
        xko.append((px.add_leaf(lf), lf.obj))
        n_ext += 1
    if not elem_src:
        raise RadiaError("Radia::Error118: no relaxable elements (apply a material first)")
    pack = InteractionPack(
        elems=pe.arrays(), ext=(px.arrays() if n_ext else None),
        elem_src=np.ascontiguousarray(np.array(elem_src, dtype=np.int32).reshape(-1, 2)),
        mat_kind=np.ascontiguousarray(np.array(mat_kind, dtype=np.int32)),
        mat=np.ascontiguousarray(np.array(mats, dtype=np.float64).reshape(-1, MAT_STRIDE)),
        mh=(np.ascontiguousarray(np.array(mh_rows, dtype=np.float64).reshape(-1, 3))
            if mh_rows else np.zeros((0, 3))),
        leaves=relax_leaves, main=mains)
    if len(_INT_CACHE) >= _SRC_CACHE_MAX:
        _INT_CACHE.pop(next(iter(_INT_CACHE)))
    _INT_CACHE[key] = (fp, pack, _m_slots(eko), _m_slots(xko), leaves + sleaves, _mat_groups(relax_leaves))
    return InteractionPack(
        elems={k: v.copy() for k, v in pack.elems.items()},
        ext=({k: v.copy() for k, v in pack.ext.items()} if pack.ext is not None else None),
        elem_src=pack.elem_src.copy(), mat_kind=pack.mat_kind.copy(), mat=pack.mat.copy(), mh=pack.mh.copy(),
        leaves=list(relax_leaves), main=list(mains))


def element_centres(pack: InteractionPack) -> np.ndarray:
    """Observation point of each element: main image of its centre."""
    e = pack.elems
    out = np.zeros((len(pack.leaves), 3))
    for i, (kind, idx) in enumerate(pack.elem_src):
        c = e["rec"][idx, 0:3] if kind == 0 else e["poly"][idx, 0:3]
        out[i] = pack.main[i].point(c)
    return out
