"""ctypes binding of libradb200.so (include/radb200.h).

The library is built in-tree by ``python -m radiacuda_b200.build``.  There is
no fallback: if the library is missing or a call fails, a RuntimeError is
raised with the library's own message.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Dict, Tuple

import numpy as np

from ._abi import GeomHolder, RelaxHolder

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "libradb200.so")

_lib = None
_vp, _dp, _i64 = C.c_void_p, C.POINTER(C.c_double), C.c_int64
# RadB200PointField: (ctx, geometry, pts, npts, what, out) -> 0
POINT_FIELD = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, _dp, _i64, C.c_int, _dp)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIBPATH):
            raise RuntimeError(
                f"radiacuda_b200: {LIBPATH} is missing -- build it with `python -m radiacuda_b200.build` "
                "(there is no CPU fallback)")
        L = C.CDLL(LIBPATH)
        L.radb200_last_error.restype = C.c_char_p
        L.radb200_kernel_launches.restype = C.c_int64
        L.radb200_field.argtypes = [_vp, _dp, _i64, C.c_int, C.c_int, _dp]
        L.radb200_field_dev.argtypes = [_vp, C.c_void_p, _i64, C.c_int, C.c_int, C.c_void_p]
        L.radb200_intrc_create.argtypes = [_vp, _vp, _vp, C.c_int, C.POINTER(C.c_int64)]
        L.radb200_intrc_free.argtypes = [_i64]
        L.radb200_intrc_create_rows.argtypes = [_vp, _vp, _vp, C.c_int, C.c_int32, C.c_int32, C.POINTER(C.c_int64)]
        L.radb200_relax_rows_step.argtypes = [_i64, C.c_void_p, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p, _dp]
        L.radb200_intrc_save.argtypes = [_i64, C.c_void_p, _i64, C.POINTER(C.c_int64)]
        L.radb200_intrc_restore.argtypes = [_vp, _vp, _vp, C.c_int, C.c_void_p, _i64, C.POINTER(C.c_int64)]
        L.radb200_intrc_size.argtypes = [_i64, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
        L.radb200_intrc_matrix.argtypes = [_i64, C.c_int, C.c_void_p]
        L.radb200_intrc_extfield.argtypes = [_i64, _dp]
        L.radb200_intrc_set_extfield.argtypes = [_i64, _dp]
        L.radb200_relax.argtypes = [_i64, C.c_int, C.c_double, C.c_int, C.c_int, C.c_double, _dp, _dp, _dp]
        L.radb200_direct_solve.argtypes = [_i64, C.c_int, C.c_double, C.c_int, _dp, _dp]
        L.radb200_lu_shift.argtypes = [_i64, _dp]
        L.radb200_adjoint_solve.argtypes = [_i64, _dp, C.c_double, C.c_int, _dp, _dp]
        L.radb200_adjoint_grad.argtypes = [_i64, _dp, _dp, _dp, _dp, _dp]
        L.radb200_field_vjp.argtypes = [_i64, _dp, _dp, _i64, C.c_int, _dp, _dp, _dp, _dp]
        L.radb200_trajectories.argtypes = [_vp, C.c_double, C.c_int, _dp, C.c_double, C.c_double, C.c_int, _dp, _dp,
                                           C.POINTER(C.c_int)]
        L.radb200_field_int.argtypes = [_vp, _dp, _dp, C.c_int, C.c_int, C.c_int, C.c_double, _dp, _dp]
        L.radb200_field_int_cb.argtypes = [_vp, POINT_FIELD, _vp, _dp, _dp, C.c_int, C.c_int, C.c_double, _dp,
                                           _dp]
        _lib = L
    return _lib


def check(rc: int, what: str):
    if rc != 0:
        msg = lib().radb200_last_error().decode(errors="replace")
        raise RuntimeError(f"{what} failed ({rc}): {msg}")


def _p(a):
    return a.ctypes.data_as(_dp) if a is not None else None


def kernel_launches() -> int:
    return int(lib().radb200_kernel_launches())


def release_cached_memory() -> None:
    """Return the device blocks kept for reuse (256 MB and more, released
    interactions and factors) to the driver.  Nothing is cached before the
    library is loaded, so this does not load it."""
    if _lib is not None:
        check(_lib.radb200_release_cached_memory(), "radb200_release_cached_memory")


def field(geom: Dict[str, np.ndarray], pts: np.ndarray, what: int, precision: int = 0) -> np.ndarray:
    g = GeomHolder(geom)
    P = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 3)
    out = np.zeros_like(P)
    if P.shape[0]:
        check(lib().radb200_field(C.cast(g.ptr, _vp), _p(P), P.shape[0], what, precision, _p(out)), "radb200_field")
    return out


def field_int(geom: Dict[str, np.ndarray], P1, P2, infinite: bool, what: int, precision: int = 0,
              abs_prec: float = 1e-3) -> Tuple[np.ndarray, np.ndarray]:
    """Integral of B (what bit 0 -> out[0:3]) and/or H (bit 1 -> out[3:6])
    along the line P1 -> P2 (finite) or through P1, P2 (infinite), T mm.
    Returns (out[6], status[6]) as radb200_field_int."""
    g = GeomHolder(geom)
    a = np.ascontiguousarray(P1, dtype=np.float64).reshape(3)
    b = np.ascontiguousarray(P2, dtype=np.float64).reshape(3)
    out, st = np.zeros(6), np.zeros(6)
    check(lib().radb200_field_int(C.cast(g.ptr, _vp), _p(a), _p(b), int(bool(infinite)), int(what), int(precision),
                                  float(abs_prec), _p(out), _p(st)), "radb200_field_int")
    return out, st


def trajectories(geom: Dict[str, np.ndarray], energy_gev: float, init: np.ndarray, y0: float, y1: float, np_: int,
                 prec=None) -> np.ndarray:
    """Electron trajectories (radb200_trajectories): init [n, 4] (x, x', z, z')
    -> [n, np_, 5] (y, x, x', z, z')."""
    g = GeomHolder(geom)
    X = np.ascontiguousarray(init, dtype=np.float64).reshape(-1, 4)
    out = np.zeros((X.shape[0], int(np_), 5))
    st = np.zeros(X.shape[0], dtype=np.int32)
    pr = None if prec is None else np.ascontiguousarray(prec, dtype=np.float64).reshape(4)
    check(lib().radb200_trajectories(C.cast(g.ptr, _vp), float(energy_gev), X.shape[0], _p(X), float(y0), float(y1),
                                     int(np_), _p(pr), _p(out), st.ctypes.data_as(C.POINTER(C.c_int))),
          "radb200_trajectories")
    return out


def field_int_cb(geom: Dict[str, np.ndarray], point_field, P1, P2, infinite: bool, what: int,
                 abs_prec: float = 1e-3) -> Tuple[np.ndarray, np.ndarray]:
    """The quadrature of field_int around ``point_field(geom_ptr, pts[n,3],
    what) -> [n,3]`` (host code, no device use)."""
    g = GeomHolder(geom)

    def cb(ctx, gp, pts, n, w, out):
        try:
            P = np.ctypeslib.as_array(pts, shape=(n, 3))
            O = np.ctypeslib.as_array(out, shape=(n, 3))
            O[:] = point_field(gp, P, w)
            return 0
        except Exception:  # reported to the library as a failed evaluation
            return 1

    fn = POINT_FIELD(cb)
    a = np.ascontiguousarray(P1, dtype=np.float64).reshape(3)
    b = np.ascontiguousarray(P2, dtype=np.float64).reshape(3)
    out, st = np.zeros(6), np.zeros(6)
    check(lib().radb200_field_int_cb(C.cast(g.ptr, _vp), fn, None, _p(a), _p(b), int(bool(infinite)), int(what),
                                     float(abs_prec), _p(out), _p(st)), "radb200_field_int_cb")
    return out, st


def field_dev(geom: Dict[str, np.ndarray], d_pts_ptr: int, npts: int, what: int, d_out_ptr: int, precision: int = 0):
    """Field with points/results already on the device (raw CUDA pointers)."""
    g = GeomHolder(geom)
    check(lib().radb200_field_dev(C.cast(g.ptr, _vp), C.c_void_p(d_pts_ptr), npts, what, precision,
                                  C.c_void_p(d_out_ptr)), "radb200_field_dev")


class NativeInteraction:
    """Owner of a device-resident interaction (radb200_intrc_*)."""

    def __init__(self, pack, storage: int = 0, state: bytes = None):
        """Assembles the interaction of pack on the device, or, given a state
        saved by save(), restores it without assembling."""
        self.pack = pack
        self.storage = storage
        self._g = GeomHolder(pack.elems)
        self._r = RelaxHolder(pack.elem_src, pack.mat_kind, pack.mat, pack.mh)
        self._x = GeomHolder(pack.ext) if pack.ext is not None else None
        h = C.c_int64(0)
        xg = C.cast(self._x.ptr, _vp) if self._x else None
        if state is None:
            check(lib().radb200_intrc_create(C.cast(self._g.ptr, _vp), C.cast(self._r.ptr, _vp), xg, storage,
                                             C.byref(h)), "radb200_intrc_create")
        else:
            buf = C.create_string_buffer(bytes(state), len(state))
            check(lib().radb200_intrc_restore(C.cast(self._g.ptr, _vp), C.cast(self._r.ptr, _vp), xg, storage, buf,
                                              len(state), C.byref(h)), "radb200_intrc_restore")
        self.handle = h.value
        self.n = pack.elem_src.shape[0]

    def save(self) -> bytes:
        """The interaction's device state (radb200_intrc_save)."""
        n = C.c_int64(0)
        check(lib().radb200_intrc_save(self.handle, None, 0, C.byref(n)), "radb200_intrc_save")
        buf = C.create_string_buffer(n.value)
        check(lib().radb200_intrc_save(self.handle, buf, n.value, C.byref(n)), "radb200_intrc_save")
        return buf.raw[:n.value]

    def free(self):
        if self.handle:
            lib().radb200_intrc_free(self.handle)
            self.handle = 0

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def matrix(self, dtype=np.float32) -> np.ndarray:
        n3 = 3 * self.n
        out = np.zeros((n3, n3), dtype=dtype)
        check(lib().radb200_intrc_matrix(self.handle, 1 if dtype == np.float64 else 0,
                                         out.ctypes.data_as(C.c_void_p)), "radb200_intrc_matrix")
        return out

    def extfield(self) -> np.ndarray:
        out = np.zeros(3 * self.n)
        check(lib().radb200_intrc_extfield(self.handle, _p(out)), "radb200_intrc_extfield")
        return out

    def relax(self, method: int, prec: float, max_iter: int, reset: bool, omega: float, M0: np.ndarray):
        M = np.ascontiguousarray(M0, dtype=np.float64).copy()
        H = np.zeros(3 * self.n)
        st = np.zeros(4)
        check(lib().radb200_relax(self.handle, method, prec, max_iter, 1 if reset else 0, omega, _p(M), _p(H), _p(st)),
              "radb200_relax")
        return M, H, st

    def direct(self, mode: int, rtol: float, max_iter: int) -> Tuple[np.ndarray, np.ndarray]:
        M = np.zeros(3 * self.n)
        st = np.zeros(4)
        check(lib().radb200_direct_solve(self.handle, mode, rtol, max_iter, _p(M), _p(st)), "radb200_direct_solve")
        return M, st

    def lu_shift(self) -> float:
        """sigma of the current factorization (A + sigma I), 0 for A itself."""
        v = C.c_double(0.0)
        check(lib().radb200_lu_shift(self.handle, C.byref(v)), "radb200_lu_shift")
        return v.value

    def adjoint_solve(self, dLdM: np.ndarray, rtol: float = 1e-12, max_iter: int = 500):
        g = np.ascontiguousarray(dLdM, dtype=np.float64)
        lam = np.zeros(3 * self.n)
        st = np.zeros(4)
        check(lib().radb200_adjoint_solve(self.handle, _p(g), rtol, max_iter, _p(lam), _p(st)),
              "radb200_adjoint_solve")
        return lam, st

    def adjoint_grad(self, lam: np.ndarray, want=("Mr", "chi", "c", "d")):
        """Per-element sensitivities through the converged solve (radb200_adjoint_grad)."""
        lam = np.ascontiguousarray(lam, dtype=np.float64)
        out = {k: np.zeros(9 * self.n if k == "chi" else 3 * self.n) for k in want}
        check(lib().radb200_adjoint_grad(self.handle, _p(lam), *[(_p(out[k]) if k in out else None)
                                                                  for k in ("Mr", "chi", "c", "d")]),
              "radb200_adjoint_grad")
        return out

    def field_vjp(self, M: np.ndarray, pts: np.ndarray, what: int, W: np.ndarray):
        """(dF/dM)^T W and the centre / dimension gradients of W.F at fixed M."""
        M = np.ascontiguousarray(M, dtype=np.float64)
        P = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 3)
        W = np.ascontiguousarray(W, dtype=np.float64).reshape(-1, 3)
        gM, gc, gd = np.zeros(3 * self.n), np.zeros(3 * self.n), np.zeros(3 * self.n)
        check(lib().radb200_field_vjp(self.handle, _p(M), _p(P), P.shape[0], what, _p(W), _p(gM), _p(gc), _p(gd)),
              "radb200_field_vjp")
        return gM, gc, gd
