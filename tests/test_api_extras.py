"""rad.ObjFullMag, rad.ObjDegFre, rad.ObjDrwAtr, rad.ObjCylMag,
rad.ObjArcPgnMag and rad.ObjCntSize: the reference's counts, sizes, errors
and return values, the same models as the reference builds (their field
through the oracle against the compiled reference module, when present), and
a relaxed model of these constructors against committed golden vectors."""
import numpy as np
import pytest

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
    # the reference's sizes: direct members of a container, 0 for one element
    assert rad.ObjCntSize(top) == 2 and rad.ObjCntSize(cnt) == 3 and rad.ObjCntSize(tet) == 0


def test_full_magnet_model_matches_reference(rad, ref):
    hr = _build(ref)
    ho = _build(rad)
    assert [ref.ObjDegFre(h) for h in hr] == [rad.ObjDegFre(h) for h in ho]
    P = np.random.default_rng(2).uniform(-15, 45, size=(30, 3)) + np.array([0.013, 0.007, 0.011])
    Br = np.array(ref.Fld(hr[0], "b", P.tolist()))
    Bo = O.field(model.pack_sources(rad._objs, ho[0], tuple(rad._rand)), P, 0)
    assert np.abs(Br - Bo).max() / np.abs(Br).max() < 1e-10


CYLINDERS = [([1.1, -0.3, 2.2], 3.0, 5.0, 12, "z", [0.1, 0.2, 1.0]), ([0.2, 0.4, -1.0], 2.0, 4.0, 7, "x", [1.0, 0.3, 0.0]),
             ([-1.0, 2.0, 0.5], 2.5, 3.0, 9, "y", [0.2, 1.0, 0.4])]


def test_cylinder_errors_and_axial_field(rad):
    for bad, code in (((0, 0, 0), 0.0, 1.0, 8), "Error089"), (((0, 0, 0), 1.0, 0.0, 8), "Error012"), \
            (((0, 0, 0), 1.0, 1.0, 0), "Error090"):
        with pytest.raises(RuntimeError, match=code):
            rad.ObjCylMag(*bad)
    # a long 64-gon prism magnetized along its axis: B at the centre is close
    # to M (1 - cos of the half-angle seen from the centre)
    rad.UtiDelAll()
    rad.FldLenRndSw("off")
    h = rad.ObjCylMag([0, 0, 0], 1.0, 200.0, 64, "z", [0, 0, 1.0])
    b = O.field(model.pack_sources(rad._objs, h, tuple(rad._rand)), np.array([[0.01, 0.007, 0.013]]), 0)[0]
    assert abs(b[2] - 100.0 / np.hypot(100.0, 1.0)) < 2e-3


def test_cylinders_match_reference(rad, ref):
    rng = np.random.default_rng(5)
    for args in CYLINDERS:
        for X in (ref, rad):
            X.UtiDelAll()
            X.FldLenRndSw("off")
        hr, ho = ref.ObjCylMag(*args), rad.ObjCylMag(*args)
        P = rng.uniform(-6, 6, size=(30, 3)) + np.array([0.0137, 0.0071, 0.0113])
        Br = np.array(ref.Fld(hr, "b", P.tolist()))
        Bo = O.field(model.pack_sources(rad._objs, ho, tuple(rad._rand)), P, 0)
        assert np.abs(Br - Bo).max() / np.abs(Br).max() < 1e-10


ARCS = [([1.0, 2.0], "z", [[3, -1], [5, -1.5], [6, 1], [3.5, 1.2]], [0.2, 2.4], 5, "nosym", [0.3, 1.0, 0.2]),
        ([1.0, 2.0], "z", [[3, -1], [5, -1.5], [6, 1], [3.5, 1.2]], [0.2, 2.4], 5, "sym", [0.3, 1.0, 0.2]),
        ([0.5, -0.3], "x", [[0, -1], [2, -1], [2, 1], [0, 1]], [0.0, 3.0], 4, "nosym", [0, 0.5, 1.0]),
        ([0.5, -0.3], "y", [[0, -1], [2, 0], [0, 1]], [-1.0, 1.5], 3, "sym", [1.0, 0.2, 0.1])]


def test_arc_structure_and_errors(rad):
    rad.UtiDelAll()
    sizes = [(rad.ObjCntSize(h), rad.ObjDegFre(h)) for h in (rad.ObjArcPgnMag(*c) for c in ARCS)]
    # 'nosym' makes one element per sector, 'sym' one element with images
    assert sizes == [(5, 15), (0, 3), (4, 12), (0, 3)]
    sq = [[1, 0], [2, 0], [2, 1], [1, 1]]
    for args, code in ((([0, 0], "w", sq, [0, 1], 2), "Error092"), (([0, 0], "z", sq, [1, 0], 2), "Error011"),
                       (([0, 0], "z", sq, [0, 1], 0), "Error090"), (([0, 0], "z", sq, [0, 3.5], 1), "Error094"),
                       (([0, 0], "z", [[-1, 0], [2, 0], [2, 1]], [0, 1], 2), "Error095")):
        with pytest.raises(RuntimeError, match=code):
            rad.ObjArcPgnMag(*args)
    with pytest.raises(RuntimeError, match="Error093"):
        rad.ObjArcPgnMag([0, 0], "z", sq, [0, 1], 2, "both")


def test_arcs_match_reference(rad, ref):
    rng = np.random.default_rng(9)
    for args in ARCS:
        for X in (ref, rad):
            X.UtiDelAll()
            X.FldLenRndSw("off")
        hr, ho = ref.ObjArcPgnMag(*args), rad.ObjArcPgnMag(*args)
        assert (ref.ObjCntSize(hr), ref.ObjDegFre(hr)) == (rad.ObjCntSize(ho), rad.ObjDegFre(ho))
        P = rng.uniform(-7, 7, size=(40, 3)) + np.array([0.0137, 0.0071, 0.0113])
        Br = np.array(ref.Fld(hr, "b", P.tolist()))
        Bo = O.field(model.pack_sources(rad._objs, ho, tuple(rad._rand)), P, 0)
        assert np.abs(Br - Bo).max() / np.abs(Br).max() < 1e-10


def test_relaxed_constructor_model_matches_reference_golden(rad):
    """Arcs ('nosym' elements carry their own rotation, 'sym' ones are
    images), an x-axis cylinder and rectangle slices with anisotropic and
    saturating materials, relaxed by the oracle's method 4 to 1e-8 like the
    reference's Solve: B agrees to 1e-8 (tests/golden/make_constructors_golden.py)."""
    import json
    import os
    import sys

    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    from make_constructors_golden import build
    from test_oracle_pin import oracle_solve

    gold = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "constructors.json")))
    h = build(rad)
    _, _, st = oracle_solve(rad, h, 1e-8, 5000)
    assert int(st[3]) == int(gold["status"][3])
    B = O.field(model.pack_sources(rad._objs, h, tuple(rad._rand)), np.array(gold["points"]), 0)
    assert np.abs(B - np.array(gold["b"])).max() / np.abs(np.array(gold["b"])).max() < 1e-8
