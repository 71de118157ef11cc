"""rad.ObjFullMag, rad.ObjDegFre and rad.ObjDrwAtr: the reference's counts
and return values, and the same model as the reference builds (its field
through the oracle against the compiled reference module, when present)."""
import numpy as np

from radiacuda_b200 import model

import oracle.oracle as O


def _build(X):
    X.UtiDelAll()
    X.FldLenRndSw("off")
    cnt = X.ObjCnt([])
    mat = X.MatLin([0.06, 0.17], [0.3, 0.2, 1.1])
    b1 = X.ObjFullMag([0.1, 0.2, 0.3], [10, 8, 6], [0.3, 0.2, 1.1], [2, 3, 1], cnt, mat, [1, 0, 0])
    b2 = X.ObjFullMag([20.1, 0.2, 0.3], [6, 6, 6], [0, 0, 1.2], [[2, 0.5], [1, 1], [3, 2.0]], cnt, 0, [0, 1, 0])
    tet = X.ObjPolyhdr([[30, 0, 0], [36, 0, 0], [30, 5, 0], [30, 0, 7]],
                       [[1, 2, 3], [1, 2, 4], [1, 3, 4], [2, 3, 4]], [0, 0, 1])
    X.ObjAddToCnt(cnt, [tet])
    X.TrfZerPerp(cnt, [0, 0, -20], [0, 0, 1])
    arc = X.ObjArcCur([0, 0, 50], [5, 8], [0, 3], 4, 10, 1.5)
    return X.ObjCnt([cnt, arc]), cnt, b1, b2, tet


def test_degrees_of_freedom_and_drawing_attributes(rad):
    top, cnt, b1, b2, tet = _build(rad)
    # the reference's counts for this model: 6 blocks with a material, a
    # polyhedron without one, 6 blocks without one, a coil; images not counted
    assert [rad.ObjDegFre(h) for h in (top, cnt, b1, b2, tet)] == [21, 21, 18, 0, 3]
    assert rad.ObjDrwAtr(b1, [0, 0, 1], 0.002) == b1
    assert rad.ObjCntSize(b1) == 6


def test_full_magnet_model_matches_reference(rad, ref):
    hr = _build(ref)
    ho = _build(rad)
    assert [ref.ObjDegFre(h) for h in hr] == [rad.ObjDegFre(h) for h in ho]
    P = np.random.default_rng(2).uniform(-15, 45, size=(30, 3)) + np.array([0.013, 0.007, 0.011])
    Br = np.array(ref.Fld(hr[0], "b", P.tolist()))
    Bo = O.field(model.pack_sources(rad._objs, ho[0], tuple(rad._rand)), P, 0)
    assert np.abs(Br - Bo).max() / np.abs(Br).max() < 1e-10
