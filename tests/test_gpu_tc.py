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
    # 1 cp.async-fed kernel, 2 TMA-fed (TF32 operands), 3 TMA-fed with scaled FP16 operands
    assert st.value in (1, 2, 3), (st.value, err.value, L.radb200_last_error())
    assert err.value < 1e-4


@pytest.mark.parametrize("ncell,ntets", [(4, 384), (6, 1200)])
def test_tf32_lu_gmres_ir_reaches_fp64_solution(cuda, rad, ncell, ntets):
    """TF32 tensor-core factors as the preconditioner of FP64 GMRES on the
    FP64 matrix: the FP64 solution to 1e-9."""
    h, body = MD.tet_mesh(rad, ncell=ncell, n_tets=ntets, chi=1000.0)
    pack = model.pack_interaction(rad._objs, h, 0, tuple(rad._rand))
    Md = O.linear_direct(pack, O.assemble(pack), O.extfield(pack))
    nat = _native.NativeInteraction(pack, 1)
    try:
        M, st = nat.direct(1, 1e-13, 200)
    finally:
        nat.free()
    assert rel_err(M, Md) < 1e-9
    assert st[0] < 1e-12


@pytest.mark.parametrize("ncell,ntets", [(4, 384), (6, 1200)])
def test_mixed_storage_near_far_solution(cuda, rad, ncell, ntets):
    """Mixed storage: FP32 blocks plus the FP64 residue of near blocks.  The
    refined solution is exact for that operator (residual 1e-12); it differs
    from the FP64 solution only by the FP32 rounding of far blocks -- M to
    1e-6 and B outside the body to 1e-8 at chi = 1000."""
    h, body = MD.tet_mesh(rad, ncell=ncell, n_tets=ntets, chi=1000.0)
    pack = model.pack_interaction(rad._objs, h, 0, tuple(rad._rand))
    N64 = O.assemble(pack)
    Md = O.linear_direct(pack, N64, O.extfield(pack))
    nat = _native.NativeInteraction(pack, 2)
    try:
        M, st = nat.direct(1, 1e-13, 200)
        Nm = nat.matrix(np.float64)
    finally:
        nat.free()
    assert st[0] < 1e-12
    assert rel_err(M, Md) < 1e-6
    # the operator: exact (FP64) near blocks, FP32-rounded far blocks
    assert np.abs(Nm - N64).max() <= 2.0 ** -23 * np.abs(N64).max()
    for lf, k in zip(pack.leaves, range(len(pack.leaves))):
        lf.obj.m = M[3 * k:3 * k + 3]
    P = MD.tet_mesh_points(500, ncell=ncell)
    src = model.pack_sources(rad._objs, h, tuple(rad._rand))
    B = O.field(src, P, 0)
    for lf, k in zip(pack.leaves, range(len(pack.leaves))):
        lf.obj.m = Md[3 * k:3 * k + 3]
    Bd = O.field(model.pack_sources(rad._objs, h, tuple(rad._rand)), P, 0)
    assert rel_err(B, Bd) < 1e-8
