"""radb200_field_noalloc: field evaluation for callers that cannot allocate.

Some callers of this library cannot call cudaMalloc -- code that runs while
another part of the process captures a CUDA graph, real-time loops that must
stay off the allocator, hosts that hand the library fixed device arenas.  The
no-alloc entry point takes every array (geometry, points, output) in device
memory and keeps its scratch in a static device array.  This test builds the
device arrays with torch, calls the entry point through the C-ABI twice in a
row and compares both results with the allocating entry point radb200_field
at the FP64 field tolerance of the other GPU tests (1e-10 relative).

Collected last on purpose (file name), so a run that stops at the first
failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

import models as MD
from radiacuda_b200 import _abi, _native, model

pytestmark = pytest.mark.gpu

_ORDER = ["trf", "rec", "rec_img", "poly", "poly_info", "face", "face_vtx", "vtx2d", "arc", "arc_img", "bkg", "bkg_img"]


def _device_geom(arrs, torch, dev):
    """RadB200Geom whose pointer fields point to device copies of arrs."""
    keep = {}
    ptr = {}
    for k in _ORDER:
        a = np.ascontiguousarray(arrs[k])
        if a.size == 0:
            ptr[k] = None
            continue
        t = torch.from_numpy(a.copy()).to(dev)
        keep[k] = t
        ptr[k] = t.data_ptr()
    dp, ip = C.POINTER(C.c_double), C.POINTER(C.c_int32)

    def P(k, typ):
        return C.cast(C.c_void_p(ptr[k]), typ) if ptr[k] else None

    g = _abi.RadB200Geom(
        arrs["trf"].shape[0], P("trf", dp),
        arrs["rec"].shape[0], P("rec", dp), P("rec_img", ip),
        arrs["poly"].shape[0], P("poly", dp), P("poly_info", ip),
        arrs["face"].shape[0], P("face", dp), P("face_vtx", ip),
        arrs["vtx2d"].shape[0], P("vtx2d", dp),
        arrs["arc"].shape[0], P("arc", dp), P("arc_img", ip),
        arrs["bkg"].shape[0], P("bkg", dp), P("bkg_img", ip),
        float(arrs["rand"][0]), float(arrs["rand"][1]), float(arrs["rand"][2]))
    return g, keep


def test_field_noalloc_matches_allocating_entry_point(cuda, rad):
    import torch

    L = _native.lib()
    L.radb200_field_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_int, C.c_void_p]
    # mixed cuboids, tetrahedra, arcs and a racetrack, plus a uniform
    # background (a source kind with no M and no inside test)
    h = rad.ObjCnt([MD.mixed_sym(rad), rad.ObjBckg([0.11, -0.07, 0.23])])
    rng = np.random.default_rng(21)
    for lf in model.collect_leaves(rad._objs, h):
        if hasattr(lf.obj, "m") and not (hasattr(lf.obj, "j") and np.any(lf.obj.j != 0)):
            lf.obj.m = rng.normal(size=3)
    arrs = model.pack_sources(rad._objs, h, tuple(rad._rand))
    g, keep = _device_geom(arrs, torch, cuda)
    P = rng.uniform(-90, 90, size=(3000, 3))
    # points inside the magnets too, so the M path (what == 2) sees both sides
    P[:200] = _inside_points(arrs, 200, rng)
    d_pts = torch.from_numpy(P).to(cuda)
    for what in (0, 1, 2):
        ref = _native.field(arrs, P, what, 0)
        for call in range(2):
            d_out = torch.full((P.shape[0], 3), float("nan"), dtype=torch.float64, device=cuda)
            rc = L.radb200_field_noalloc(C.cast(C.byref(g), C.c_void_p), C.c_void_p(d_pts.data_ptr()), P.shape[0], what,
                                         C.c_void_p(d_out.data_ptr()))
            _native.check(rc, "radb200_field_noalloc")
            got = d_out.cpu().numpy()
            if what == 2:
                assert np.array_equal(got, ref), (what, call)
                assert np.abs(ref).max() > 0
                continue
            err = np.abs(got - ref).max() / np.abs(ref).max()
            assert err < 1e-10, (what, call, err)


def _inside_points(arrs, n, rng):
    """Points inside the cuboids (centre + a fraction of the half widths),
    mapped by each cuboid's first image."""
    rec, img, trf = arrs["rec"], arrs["rec_img"], arrs["trf"]
    out = []
    for k in range(n):
        i = k % rec.shape[0]
        if np.any(rec[i, 9:12] != 0):
            i = 0
        q = rec[i, 0:3] + rng.uniform(-0.4, 0.4, 3) * rec[i, 3:6]
        T = trf[img[i, 0]]
        M = np.linalg.inv(T[0:9].reshape(3, 3))
        out.append(M @ q + T[9:12])
    return np.array(out)


def test_field_noalloc_rejects_oversized_calls(cuda, rad):
    import torch

    L = _native.lib()
    L.radb200_field_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_int, C.c_void_p]
    h = MD.magnet_array(rad, nside=2, div=1)
    arrs = model.pack_sources(rad._objs, h, tuple(rad._rand))
    g, keep = _device_geom(arrs, torch, cuda)
    n = 16385
    d_pts = torch.zeros((n, 3), dtype=torch.float64, device=cuda)
    d_out = torch.zeros((n, 3), dtype=torch.float64, device=cuda)
    rc = L.radb200_field_noalloc(C.cast(C.byref(g), C.c_void_p), C.c_void_p(d_pts.data_ptr()), n, 0,
                                 C.c_void_p(d_out.data_ptr()))
    assert rc == -1
    assert b"16384" in L.radb200_last_error()
