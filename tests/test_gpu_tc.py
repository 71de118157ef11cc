"""The tcgen05 TF32 GEMM of the LU: self-test against the CUDA-core GEMM, and
the mixed-precision direct solve reaching the FP64 solution (GMRES-IR)."""
import ctypes as C

import numpy as np
import pytest

import models as MD
from radiacuda_b200 import _native, model
from util import rel_err

import oracle.oracle as O

pytestmark = pytest.mark.gpu


def test_tensor_core_selftest_passes(cuda):
    L = _native.lib()
    L.radb200_tc_selftest.argtypes = [C.POINTER(C.c_int), C.POINTER(C.c_double)]
    st, err = C.c_int(-1), C.c_double(-1)
    _native.check(L.radb200_tc_selftest(C.byref(st), C.byref(err)), "tc selftest")
    assert st.value in (1, 2), (st.value, err.value, L.radb200_last_error())
    assert err.value < 1e-4


@pytest.mark.parametrize("ncell,ntets", [(4, 384), (6, 1200)])
def test_tf32_lu_gmres_ir_reaches_fp64_solution(cuda, rad, ncell, ntets):
    h, body = MD.tet_mesh(rad, ncell=ncell, n_tets=ntets, chi=1000.0)
    pack = model.pack_interaction(rad._objs, h, 0, tuple(rad._rand))
    Md = O.linear_direct(pack, O.assemble(pack), O.extfield(pack))
    nat = _native.NativeInteraction(pack, 2)
    try:
        M, st = nat.direct(1, 1e-13, 200)
    finally:
        nat.free()
    assert rel_err(M, Md) < 1e-9
    assert st[0] < 1e-12
