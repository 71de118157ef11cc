"""CPU-side checks of the boundary: the library loads without a GPU and exports
every entry point include/radb200.h declares; host-side packing logic."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from radiacuda_b200 import _native, model

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "radb200.h")).read()
    return sorted(set(re.findall(r"RADB200_API\s+[\w\s\*]+?\b(radb200_\w+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    L = _native.lib()
    names = _declared()
    assert len(names) >= 17
    for n in names:
        assert hasattr(L, n), n
    out = subprocess.run(["nm", "-D", "--defined-only", _native.LIBPATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (radb200_\w+)", out))
    assert set(names) <= exported


def test_version_and_error_string():
    L = _native.lib()
    assert L.radb200_version() == 100
    assert isinstance(L.radb200_last_error(), bytes)


def test_bad_handle_is_an_error_not_a_crash():
    L = _native.lib()
    assert L.radb200_intrc_free(ctypes.c_int64(987654)) == -4


def test_transform_products_and_images():
    t1 = model.trf_plane_sym([0, 0, 0], [1, 0, 0])
    t2 = model.trf_field_inversion() @ model.trf_plane_sym([0, 0, 0], [0, 0, 1])
    ims = model.images_of([(2, t1), (2, t2)])
    assert len(ims) == 4
    assert np.allclose(ims[0].M, np.eye(3)) and ims[0].s == 1.0
    p = np.array([1.0, 2.0, 3.0])
    assert np.allclose(ims[3].point(p), [-1, 2, -3]) and ims[3].s == -1.0
    r = model.trf_rotation([1, 2, 3], [0, 0, 1], np.pi / 2)
    assert np.allclose(r.point([2, 2, 3]), [1, 3, 3])
    assert np.allclose(r.Minv @ r.M, np.eye(3))


def test_polyhedron_faces_are_outward_and_ccw():
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], float)
    for faces in ([[0, 1, 2], [0, 3, 1], [1, 3, 2], [2, 3, 0]], [[0, 2, 1], [0, 1, 3], [1, 2, 3], [2, 0, 3]]):
        p = model.Polyhedron(v, faces, [0, 0, 1])
        for k, f in enumerate(p.face_rec):
            R = f[0:9].reshape(3, 3)
            n = R[2]
            # outward: centre on the inner side, z of the face plane > z of the centre
            assert (R @ p.centre)[2] < f[9]
            pts = p.face_v2d[k]
            area = 0.5 * sum(pts[i][0] * pts[(i + 1) % 3][1] - pts[(i + 1) % 3][0] * pts[i][1] for i in range(3))
            assert area > 0
            assert abs(np.linalg.norm(n) - 1) < 1e-14


def test_divmag_matches_reference_geometry(ref, rad):
    for R in (ref, rad):
        R.UtiDelAll()
        R.FldLenRndSw("off")
    a = ref.ObjRecMag([1, 2, 3], [4, 5, 6], [0.1, 0.2, 0.3])
    ref.ObjDivMag(a, [[3, 2.0], [2, 0.5], [1, 1]])
    b = rad.ObjRecMag([1, 2, 3], [4, 5, 6], [0.1, 0.2, 0.3])
    rad.ObjDivMag(b, [[3, 2.0], [2, 0.5], [1, 1]])
    assert np.allclose(np.array(ref.ObjM(a), dtype=object)[:, 0].tolist(),
                       np.array(rad.ObjM(b), dtype=object)[:, 0].tolist(), atol=1e-12)


def test_objm_images_match_reference(ref, rad):
    out = []
    for R in (ref, rad):
        R.UtiDelAll()
        R.FldLenRndSw("off")
        a = R.ObjRecMag([1, 2, 3], [1, 1, 1], [0.1, 0.2, 0.3])
        b = R.ObjRecMag([5, 2, 3], [1, 1, 1], [0.4, 0.5, 0.6])
        g = R.ObjCnt([a, b])
        R.TrfZerPerp(g, [0, 0, 0], [1, 0, 0])
        R.TrfZerPara(g, [0, 0, 0], [0, 0, 1])
        R.TrfOrnt(b, R.TrfRot([0, 0, 0], [0, 0, 1], 0.5))
        out.append(np.array(R.ObjM(g), dtype=float))
    assert out[0].shape == out[1].shape
    assert np.allclose(out[0], out[1], atol=1e-12)


def test_api_errors_follow_reference(rad):
    rad.UtiDelAll()
    with pytest.raises(RuntimeError):
        rad.ObjRecMag([0, 0, 0], [-1, 1, 1])
    with pytest.raises(RuntimeError):
        rad.MatLin([0.1, 0.2], [0, 0, 0])
    with pytest.raises(RuntimeError):
        rad.ObjArcCur([0, 0, 0], [2, 1], [0, 1], 1, 4, 1.0)
    m = rad.ObjRecMag([0, 0, 0], [1, 1, 1], [0, 0, 0])
    with pytest.raises(RuntimeError):
        rad.MatApl(m, rad.MatLin([0.1, 0.2], 1.2))   # easy axis from a zero magnetization
