"""ctypes mirror of the structs in include/radb200.h.

Builds RadB200Geom / RadB200Relax views over numpy arrays produced by
``model.Packed.arrays()``.  The returned holder keeps the arrays alive for as
long as the struct is in use.
"""
from __future__ import annotations

import ctypes as C
from typing import Dict, Optional

import numpy as np

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


class RadB200Geom(C.Structure):
    _fields_ = [
        ("n_trf", C.c_int32), ("trf", _dp),
        ("n_rec", C.c_int32), ("rec", _dp), ("rec_img", _ip),
        ("n_poly", C.c_int32), ("poly", _dp), ("poly_info", _ip),
        ("n_face", C.c_int32), ("face", _dp), ("face_vtx", _ip),
        ("n_vtx", C.c_int32), ("vtx2d", _dp),
        ("n_arc", C.c_int32), ("arc", _dp), ("arc_img", _ip),
        ("n_bkg", C.c_int32), ("bkg", _dp), ("bkg_img", _ip),
        ("abs_rand", C.c_double), ("rel_rand", C.c_double), ("zero_rand", C.c_double),
    ]


class RadB200Relax(C.Structure):
    _fields_ = [
        ("n_elem", C.c_int32), ("elem_src", _ip), ("mat_kind", _ip), ("mat", _dp),
        ("n_mh", C.c_int32), ("mh_table", _dp),
    ]


def _d(a: np.ndarray):
    return a.ctypes.data_as(_dp) if a.size else None


def _i(a: np.ndarray):
    return a.ctypes.data_as(_ip) if a.size else None


class GeomHolder:
    def __init__(self, arrs: Dict[str, np.ndarray]):
        self.arrs = {k: np.ascontiguousarray(v) for k, v in arrs.items()}
        a = self.arrs
        self.struct = RadB200Geom(
            a["trf"].shape[0], _d(a["trf"]),
            a["rec"].shape[0], _d(a["rec"]), _i(a["rec_img"]),
            a["poly"].shape[0], _d(a["poly"]), _i(a["poly_info"]),
            a["face"].shape[0], _d(a["face"]), _i(a["face_vtx"]),
            a["vtx2d"].shape[0], _d(a["vtx2d"]),
            a["arc"].shape[0], _d(a["arc"]), _i(a["arc_img"]),
            a["bkg"].shape[0], _d(a["bkg"]), _i(a["bkg_img"]),
            float(a["rand"][0]), float(a["rand"][1]), float(a["rand"][2]))

    @property
    def ptr(self):
        return C.byref(self.struct)


class RelaxHolder:
    def __init__(self, elem_src: np.ndarray, mat_kind: np.ndarray, mat: np.ndarray,
                 mh: Optional[np.ndarray] = None):
        self.elem_src = np.ascontiguousarray(elem_src, dtype=np.int32)
        self.mat_kind = np.ascontiguousarray(mat_kind, dtype=np.int32)
        self.mat = np.ascontiguousarray(mat, dtype=np.float64)
        self.mh = np.ascontiguousarray(mh if mh is not None else np.zeros((0, 3)), dtype=np.float64)
        self.struct = RadB200Relax(self.elem_src.shape[0], _i(self.elem_src), _i(self.mat_kind),
                                   _d(self.mat), self.mh.shape[0], _d(self.mh))

    @property
    def ptr(self):
        return C.byref(self.struct)
