"""rad.ObjMltExtPgn and rad.ObjMltExtRtg against the reference's golden vectors
(tests/golden/make_mltextpgn_golden.py): the same pieces and the same field,
through the CPU oracle on the packed geometry and through the device."""
import json
import os

import numpy as np
import pytest

from radiacuda_b200 import model

import oracle.oracle as O

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "mltextpgn.json")))


def _build(rad, case):
    rad.UtiDelAll()
    rad.FldLenRndSw("off")
    if "layers" in case:
        return rad.ObjMltExtRtg(case["layers"], case["M"])
    return rad.ObjMltExtPgn(case["slices"], case["M"])


def _pieces(rad, h):
    return rad.ObjCntSize(h)


def _rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / np.abs(np.asarray(b)).max())


@pytest.mark.parametrize("name", sorted(GOLD))
def test_pieces_and_field_match_reference(rad, name):
    c = GOLD[name]
    h = _build(rad, c)
    assert _pieces(rad, h) == c["pieces"]
    g = model.pack_sources(rad._objs, h, tuple(rad._rand))
    assert _rel(O.field(g, np.array(c["points"]), 0), c["b"]) < 1e-10


def test_example04_field_inside_is_two_thirds(rad):
    """A uniformly magnetized sphere (M = 1 T along x) has B = 2/3 T inside;
    the 15 x 15 polyhedral sphere of the reference's example 4 comes within
    0.1%, at the reference's own value."""
    c = GOLD["example04_sphere"]
    h = _build(rad, c)
    g = model.pack_sources(rad._objs, h, tuple(rad._rand))
    b = O.field(g, np.array([[0.001, 0.0007, 0.0013]]), 0)[0]
    assert abs(b[0] - 2.0 / 3.0) < 1e-3 and abs(b[1]) < 1e-6 and abs(b[2]) < 1e-6
    assert abs(b[0] - c["b"][40][0]) < 1e-12


@pytest.mark.parametrize("name", ["waist", "cone", "square_to_segment"])
def test_slice_order_does_not_change_the_solid(rad, name):
    """The same slices listed top to bottom describe the same solid, so the
    field is the same (the reference builds another solid from decreasing
    attitudes)."""
    c = GOLD[name]
    P = np.array(c["points"])
    h = _build(rad, c)
    b_up = O.field(model.pack_sources(rad._objs, h, tuple(rad._rand)), P, 0)
    h = _build(rad, dict(c, slices=c["slices"][::-1]))
    b_down = O.field(model.pack_sources(rad._objs, h, tuple(rad._rand)), P, 0)
    assert _rel(b_down, b_up) < 1e-12


def test_argument_errors(rad):
    with pytest.raises(RuntimeError, match="Error064"):
        rad.ObjMltExtRtg([[[0, 0, 0], [1, 1]], [[0, 0, 1], [0, 0]]])
    with pytest.raises(RuntimeError, match="Error063"):
        rad.ObjMltExtRtg([[[0, 0, 0], [1, 1]]])
    sq = [[-1, -1], [1, -1], [1, 1], [-1, 1]]
    with pytest.raises(RuntimeError, match="Error063"):
        rad.ObjMltExtPgn([[sq, 0.0]])
    with pytest.raises(RuntimeError, match="Error063"):
        rad.ObjMltExtPgn([[sq, 0.0], [sq, 1.0], [sq, 0.5]])
    with pytest.raises(RuntimeError, match="Error063"):
        rad.ObjMltExtPgn([[sq, 0.0], [sq, 0.0]])
    with pytest.raises(RuntimeError, match="Error111"):
        rad.ObjMltExtPgn([[[[0, 0], [2, 0], [0.5, 0.5], [0, 2]], 0.0], [sq, 1.0]])
    with pytest.raises(RuntimeError, match="Error063"):
        rad.ObjMltExtPgn([[[[0, 0]], 0.0], [[[0, 0], [1, 0]], 1.0], [sq, 2.0]])
    with pytest.raises(RuntimeError, match="Error063"):
        rad.ObjMltExtPgn([[[[0, 0]], 0.0], [[[1, 1]], 1.0]])


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(GOLD))
def test_device_field_matches_reference(rad, cuda, name):
    c = GOLD[name]
    h = _build(rad, c)
    assert _rel(rad.Fld(h, "b", c["points"]), c["b"]) < 1e-9


def test_crease_rule_on_convex_flat_and_reflex_slices(rad):
    """The piece rule on its own: a section of the outer slices strictly
    inside the middle one is a convex crease, equal to it is flat, and
    outside it is reflex (the two latter end a piece)."""
    from radiacuda_b200.rad import _strictly_convex_crease

    sq = lambda a: np.array([[-a, -a], [a, -a], [a, a], [-a, a]], dtype=float)
    tol = 1e-8
    assert _strictly_convex_crease(sq(1.0), sq(2.0), sq(1.0), 0.0, 1.0, 2.0, tol)        # bulge
    assert not _strictly_convex_crease(sq(1.0), sq(1.5), sq(2.0), 0.0, 1.0, 2.0, tol)    # straight taper
    assert not _strictly_convex_crease(sq(2.0), sq(1.0), sq(2.0), 0.0, 1.0, 2.0, tol)    # waist
    assert _strictly_convex_crease(sq(1.0), sq(1.6), sq(2.0), 0.0, 1.0, 2.0, tol)        # widening less fast
    # the middle slice only partly outside the hull section: reflex at one edge
    assert not _strictly_convex_crease(sq(1.0), sq(1.4) + [0.5, 0.0], sq(1.0), 0.0, 1.0, 2.0, tol)


def test_finely_sliced_sphere_is_one_polyhedron(rad):
    import math

    rad.UtiDelAll()
    rad.FldLenRndSw("off")
    nz, nphi = 40, 24
    sl = [[[[0.0, 0.0]], -1.0]]
    for i in range(1, nz):
        z = -1.0 + 2.0 * i / nz
        ct = math.sqrt(1.0 - z * z)
        sl.append([[[ct * math.cos(2 * math.pi * k / nphi), ct * math.sin(2 * math.pi * k / nphi)] for k in range(nphi)], z])
    sl.append([[[0.0, 0.0]], 1.0])
    h = rad.ObjMltExtPgn(sl, [0.0, 0.0, 1.0])
    assert rad.ObjCntSize(h) == 0
    b = O.field(model.pack_sources(rad._objs, h, tuple(rad._rand)), np.array([[0.01, 0.02, 0.03]]), 0)[0]
    assert abs(b[2] - 2.0 / 3.0) < 5e-3
