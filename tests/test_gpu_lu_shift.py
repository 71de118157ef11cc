"""The direct solve when an unpivoted LU pivot vanishes.

Three touching 10 mm cubes in a row; the first has isotropic susceptibility
-3 (unphysical), so its self block I - chi N_ii is zero up to rounding (a
cube's self demagnetization at its centre is N_ii = -I/3), while the coupled
system stays solvable.  The factorization meets a pivot below 1e-12 of the
largest |A_ii| in the first block, refactors A + sigma I, and FP64 GMRES on A
with the shifted factors as preconditioner must reach the oracle's pivoted
dense solution (numpy, FP64) in both modes.  A model of physical materials
keeps sigma = 0.
"""
import numpy as np
import pytest

from oracle import oracle as O


def _cubes(rad, chis):
    import models as MD
    MD.reset(rad)
    parts = []
    for i, chi in enumerate(chis):
        b = rad.ObjRecMag([10.0 * i, 0.0, 0.0], [10.0, 10.0, 10.0], [0.0, 0.0, 0.0])
        rad.MatApl(b, rad.MatLin([chi, chi], [0.1, 0.3, 0.5]))
        parts.append(b)
    return rad.ObjCnt(parts)


def _solve(rad, h, mode):
    from radiacuda_b200 import _native, model
    pack = model.pack_interaction(rad._objs, h, 0, tuple(rad._rand))
    nat = _native.NativeInteraction(pack, storage=1)
    try:
        M, st = nat.direct(mode, 1e-13, 200)
        sigma = nat.lu_shift()
    finally:
        nat.free()
    Md = O.linear_direct(pack, O.assemble(pack), O.extfield(pack))
    return M, st, sigma, Md


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [0, 1])
def test_vanishing_pivot_refactors_shifted_and_gmres_reaches_the_solution(cuda, rad, mode):
    h = _cubes(rad, (-3.0, 1.0, 1.0))
    M, st, sigma, Md = _solve(rad, h, mode)
    assert sigma > 0.0
    assert st[0] <= 1e-12, st
    assert np.abs(M - Md).max() <= 1e-9 * np.abs(Md).max(), (M, Md)


@pytest.mark.gpu
def test_physical_materials_need_no_shift(cuda, rad):
    h = _cubes(rad, (1000.0, 1.0, 0.05))
    M, st, sigma, Md = _solve(rad, h, 1)
    assert sigma == 0.0
    assert st[0] <= 1e-12, st
    assert np.abs(M - Md).max() <= 1e-9 * np.abs(Md).max()
