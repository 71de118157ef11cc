"""Python driver of the C oracle (oracle/radia_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, always as the checker.  The product package
never imports this module.

Functions take the packed arrays produced by ``radiacuda_b200.model`` (the
same arrays the CUDA library receives) and return numpy results computed on
the CPU in FP64.  Parity of the oracle with the reference is pinned by
tests/test_oracle_pin.py (against the compiled reference module) and by the
golden vectors under tests/golden/.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from radiacuda_b200._abi import GeomHolder, RelaxHolder

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
SRC = os.path.join(HERE, "radia_oracle.c")


def build(force: bool = False) -> str:
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(SRC):
        subprocess.check_call(["gcc", "-O2", "-fPIC", "-shared", "-fno-fast-math", "-ffp-contract=off",
                               "-o", LIB, SRC, "-lm"])
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB)
        vp, dp, fp = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_float)
        L.orc_field.argtypes = [vp, dp, C.c_int64, C.c_int, dp]
        L.orc_assemble.argtypes = [vp, vp, dp]
        L.orc_extfield.argtypes = [vp, vp, vp, dp]
        L.orc_relax_m4.argtypes = [vp, dp, fp, dp, C.c_double, C.c_int, C.c_int, dp, dp, dp]
        L.orc_material_m.argtypes = [vp, C.c_int, dp, dp]
        L.orc_material_dmdh.argtypes = [vp, C.c_int, dp, dp]
        L.orc_material_m.restype = None
        L.orc_material_dmdh.restype = None
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def field(geom_arrays, pts, what: int = 0) -> np.ndarray:
    g = GeomHolder(geom_arrays)
    pts = np.ascontiguousarray(np.asarray(pts, dtype=np.float64).reshape(-1, 3))
    out = np.zeros_like(pts)
    lib().orc_field(C.cast(g.ptr, C.c_void_p), _p(pts), pts.shape[0], what, _p(out))
    return out


def assemble(pack) -> np.ndarray:
    g = GeomHolder(pack.elems)
    r = RelaxHolder(pack.elem_src, pack.mat_kind, pack.mat, pack.mh)
    n = pack.elem_src.shape[0]
    N = np.zeros((3 * n, 3 * n))
    lib().orc_assemble(C.cast(g.ptr, C.c_void_p), C.cast(r.ptr, C.c_void_p), _p(N))
    return N


def extfield(pack) -> np.ndarray:
    n = pack.elem_src.shape[0]
    H = np.zeros(3 * n)
    if pack.ext is None:
        return H
    g = GeomHolder(pack.elems)
    x = GeomHolder(pack.ext)
    r = RelaxHolder(pack.elem_src, pack.mat_kind, pack.mat, pack.mh)
    lib().orc_extfield(C.cast(g.ptr, C.c_void_p), C.cast(r.ptr, C.c_void_p), C.cast(x.ptr, C.c_void_p), _p(H))
    return H


def relax_m4(pack, N, Hext, prec, max_iter, M0=None):
    """Method-4 Gauss-Seidel on N (float32 or float64 array)."""
    r = RelaxHolder(pack.elem_src, pack.mat_kind, pack.mat, pack.mh)
    n = pack.elem_src.shape[0]
    M = np.zeros(3 * n) if M0 is None else np.array(M0, dtype=np.float64)
    H = np.zeros(3 * n)
    st = np.zeros(4)
    Hext = np.ascontiguousarray(Hext, dtype=np.float64)
    if N.dtype == np.float32:
        N = np.ascontiguousarray(N)
        lib().orc_relax_m4(C.cast(r.ptr, C.c_void_p), None, N.ctypes.data_as(C.POINTER(C.c_float)), _p(Hext),
                           prec, max_iter, 1 if M0 is None else 0, _p(M), _p(H), _p(st))
    else:
        N = np.ascontiguousarray(N, dtype=np.float64)
        lib().orc_relax_m4(C.cast(r.ptr, C.c_void_p), _p(N), None, _p(Hext),
                           prec, max_iter, 1 if M0 is None else 0, _p(M), _p(H), _p(st))
    return M, H, st


def material_m(pack, e, H):
    r = RelaxHolder(pack.elem_src, pack.mat_kind, pack.mat, pack.mh)
    H = np.ascontiguousarray(H, dtype=np.float64)
    M = np.zeros(3)
    lib().orc_material_m(C.cast(r.ptr, C.c_void_p), e, _p(H), _p(M))
    return M


def material_dmdh(pack, e, H):
    r = RelaxHolder(pack.elem_src, pack.mat_kind, pack.mat, pack.mh)
    H = np.ascontiguousarray(H, dtype=np.float64)
    D = np.zeros(9)
    lib().orc_material_dmdh(C.cast(r.ptr, C.c_void_p), e, _p(H), _p(D))
    return D.reshape(3, 3)


def linear_direct(pack, N, Hext):
    """FP64 dense solve of (I - X N) M = X H_ext + Mr for linear materials."""
    n = pack.elem_src.shape[0]
    X = np.zeros((3 * n, 3 * n))
    Mr = np.zeros(3 * n)
    for e in range(n):
        X[3 * e:3 * e + 3, 3 * e:3 * e + 3] = pack.mat[e, 0:9].reshape(3, 3)
        Mr[3 * e:3 * e + 3] = pack.mat[e, 9:12]
    A = np.eye(3 * n) - X @ N
    return np.linalg.solve(A, X @ Hext + Mr)
