"""Radia's own Python module with this library as its GPU plugin.

``radiacuda_b200/shim/Makefile`` compiles the reference core sources,
unchanged, with ``RADIA_WITH_CUDA`` and ``shim/radgpu_b200.cpp`` in place of
the reference's GPU plugin, into ``shim/_ref/radia<EXT>``.  In that module
``rad.RlxPre(obj, use_gpu=True)``, ``rad.RlxAuto(im, prec, iters, 9 | 11)``
and ``rad.Fld(obj, 'b', pts, use_gpu=True)`` run on libradb200, exactly where
the reference's CUDA build runs its own kernels (radintrc.cpp:731-805,
radapl2.cpp:1401-1445, radentry.cpp:1073-1134).

``load()`` imports that module; ``direct_solve`` reaches the device direct
solve of a linear interaction, which the reference has no GPU method for.
"""
from __future__ import annotations

import ctypes
import importlib
import os
import sys

import numpy as np

MODULE_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "shim", "_ref")

# "tf32" (the ABI's name, RADB200_LU_TF32) and "mixed" select the FP32 factors
# with tensor-core updates (FP16 or TF32 operands, whichever passed the self-test)
_LU_MODES = {"f64": 0, "tf32": 1, "mixed": 1}


def module_path() -> str:
    import sysconfig
    return os.path.join(MODULE_DIR, "radia" + sysconfig.get_config_var("EXT_SUFFIX"))


def load():
    """Import Radia's module built with this plugin (raises if it is not built
    or if another ``radia`` module was imported first)."""
    path = module_path()
    if not os.path.exists(path):
        raise ImportError(f"{path} is not built: run radiacuda_b200/shim/Makefile (build())")
    mod = sys.modules.get("radia")
    if mod is not None:
        if os.path.realpath(getattr(mod, "__file__", "")) != os.path.realpath(path):
            raise ImportError(f"another radia module is already imported: {mod.__file__}")
        return mod
    sys.path.insert(0, MODULE_DIR)
    try:
        return importlib.import_module("radia")
    finally:
        sys.path.remove(MODULE_DIR)


def direct_solve(intrc: int, mode: str = "tf32", rtol: float = 1e-13, max_iter: int = 60) -> np.ndarray:
    """Device direct solve (radb200_direct_solve) of the interaction ``intrc``
    returned by ``rad.RlxPre``; magnetizations are written into the elements
    as a relaxation would.  Returns [relative residual, refinement iterations,
    factor seconds, total seconds]; raises RuntimeError on failure."""
    lib = ctypes.CDLL(module_path())
    fn = lib.radB200_DirectSolve
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    st = np.zeros(4)
    rc = fn(int(intrc), _LU_MODES[mode], float(rtol), int(max_iter), st.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    if rc != 0:
        from . import _native
        raise RuntimeError(f"radB200_DirectSolve failed ({rc}): {_native.lib().radb200_last_error().decode()}")
    return st
