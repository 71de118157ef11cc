"""Field integrals along straight lines (rad.FldInt, radb200_field_int).

Golden values come from the reference's own FldInt (tests/golden/fldint.json,
made by tests/golden/make_fldint_golden.py).  Where the reference's answer is
not the field integral -- finite lines crossing magnets (its per-element
Newton sums stop early at the field jumps) and infinite lines through
polyhedra (its polygon formula assumes the line misses the body,
cpp/src/core/radexpgn.cpp:704) -- the golden file also holds the reference's
own finite integrals summed over sub-segments cut at every element boundary
("value_split"), and those are compared instead.

CPU tests run the library's quadrature (radb200_field_int_cb) around the
oracle's point field; GPU tests call rad.FldInt, i.e. the device field.
"""
import ctypes as C
import json
import os

import numpy as np
import pytest

import models as MD
from radiacuda_b200 import _native, model

import oracle.oracle as O
from oracle.fldint_oracle import field_int_fin

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "fldint.json")))
FINE = 1e-9


def tet_given(R, seed=77):
    h, body = MD.tet_mesh(R, ncell=3, n_tets=150, chi=5.0)
    rng = np.random.default_rng(seed)
    for t in R.ObjCntStuf(body):
        R.ObjSetM(t, rng.normal(scale=0.6, size=3).tolist())
    return h


BUILDERS = {
    "array_given": lambda R: MD.magnet_array(R, nside=2, div=2),
    "array_relaxed": lambda R: MD.magnet_array(R, nside=2, div=2),
    "tet_given": tet_given,
    "tet_relaxed": lambda R: MD.tet_mesh(R, ncell=3, n_tets=150, chi=5.0)[0],
    "sym_given": MD.sym_blocks,
    "dipole_relaxed": lambda R: MD.iron_dipole(R, n_target=300),
    "undulator_given": lambda R: MD.undulator(R, nper_row=8, div=1)[0],
}
GIVEN = sorted(k for k in BUILDERS if k.endswith("_given"))
RELAXED = sorted(k for k in BUILDERS if k.endswith("_relaxed"))


def oracle_point_field(gp, P, what):
    out = np.zeros_like(P)
    O.lib().orc_field(C.c_void_p(gp), P.ctypes.data_as(C.POINTER(C.c_double)), P.shape[0], what,
                      out.ctypes.data_as(C.POINTER(C.c_double)))
    return out


def _target(ln):
    """(mode, P1, P2, expected) for a golden line: the reference's value, or
    its split sum (an infinite one over the finite segment it covers)."""
    if "value_split" not in ln:
        return ln["mode"], ln["P1"], ln["P2"], np.array(ln["value"])
    a, b = np.array(ln["P1"]), np.array(ln["P2"])
    if ln["mode"] == "inf":
        u = (b - a) / np.linalg.norm(b - a)
        a, b = a - ln["split_half"] * u, a + ln["split_half"] * u
        return "fin", a.tolist(), b.tolist(), np.array(ln["value_split"])
    return "fin", ln["P1"], ln["P2"], np.array(ln["value_split"])


def _tol(name, ref, prc):
    # reference analytic / converged values: quadrature and rounding; relaxed
    # models carry the relaxation's own agreement (5e-6 linear, 5e-5 saturating)
    rel = 1e-9 if name.endswith("_given") else (5e-5 if name.startswith("dipole") else 5e-6)
    return 5e-8 + max(prc, 1e-9) * 10 + rel * np.abs(ref).max()


def _relax_on_oracle(rad, h):
    pack = model.pack_interaction(rad._objs, h, 0, tuple(rad._rand))
    M, _, _ = O.relax_m4(pack, O.assemble(pack).astype(np.float32), O.extfield(pack), 1e-10, 5000)
    for e, lf in enumerate(pack.leaves):
        lf.obj.m = M[3 * e:3 * e + 3].copy()


# ---------------------------------------------------------------------------
# CPU: argument handling, component layouts, the quadrature on the oracle field
# ---------------------------------------------------------------------------
def test_fldint_argument_errors(rad):
    h = MD.magnet_array(rad, nside=2, div=2)
    with pytest.raises(Exception, match="Error033"):
        rad.FldInt(h, "half", "ib", [0, 0, 0], [1, 0, 0])
    with pytest.raises(Exception, match="Error032"):
        rad.FldInt(h, "inf", "xq", [0, 0, 0], [1, 0, 0])
    with pytest.raises(Exception, match="Error057"):
        rad.FldCmpPrc("PrcBInt=1e-6")
    with pytest.raises(Exception):
        rad.FldCmpCrt(1e-4, 1e-3, 0.0, 1, 1, 1)


@pytest.mark.parametrize("fid", sorted(GOLD["ids"]["values"]))
def test_component_layout_matches_reference(rad, fid):
    """Values and order of each id string (radsend.cpp:888-1003), from the
    B and H integrals of the golden line."""
    ib, ih, items = rad._fldint_items(fid)
    ref = GOLD["ids"]["values"][fid]
    ref = [ref] if isinstance(ref, float) else list(ref)
    full = {ln["id"]: np.array(ln["value"]) for ln in GOLD["cases"]["array_given"]["lines"][:2]}
    vals = []
    for q, comp in items:
        v = full["ib" if q == "b" else "ih"]
        vals.extend(v if comp is None else v[comp:comp + 1])
    assert len(vals) == len(ref)
    assert np.allclose(vals, ref, rtol=0, atol=1e-14)
    assert ib or ih


def test_quadrature_exact_for_smooth_fields():
    """The Gauss-Kronrod driver on an empty geometry with a polynomial and an
    analytic point field: finite integrals exact to rounding."""
    empty = model.Packed().arrays()
    P1, P2 = np.array([0.3, -1.0, 2.0]), np.array([4.3, 2.0, 2.0])
    L = np.linalg.norm(P2 - P1)

    def fld(gp, P, w):
        t = np.linalg.norm(P - P1[None, :], axis=1)
        return np.stack([t ** 5, np.sin(t), np.exp(-t)], axis=1) * (1.0 if w == 0 else 2.0)

    out, st = _native.field_int_cb(empty, fld, P1, P2, False, 3, 1e-13)
    exact = np.array([L ** 6 / 6, 1 - np.cos(L), 1 - np.exp(-L)])
    assert np.allclose(out[:3], exact, rtol=1e-13, atol=1e-13)
    assert np.allclose(out[3:], 2 * exact, rtol=1e-13, atol=1e-13)
    assert st[4] >= 1


def test_zero_length_and_degenerate_lines():
    g = model.Packed().arrays()
    out, st = _native.field_int_cb(g, lambda gp, P, w: np.ones_like(P), [1, 2, 3], [1, 2, 3], False, 1)
    assert np.all(out == 0) and st[4] == 1
    with pytest.raises(RuntimeError, match="coincide"):
        _native.field_int_cb(g, lambda gp, P, w: np.ones_like(P), [1, 2, 3], [1, 2, 3], True, 1)


@pytest.mark.parametrize("name", GIVEN + RELAXED)
def test_quadrature_on_oracle_field_matches_reference(rad, name):
    h = BUILDERS[name](rad)
    if name in RELAXED:
        _relax_on_oracle(rad, h)
    g = model.pack_sources(rad._objs, h, tuple(rad._rand))
    for ln in GOLD["cases"][name]["lines"]:
        mode, a, b, ref = _target(ln)
        what = 1 if "b" in ln["id"] else 2
        out, st = _native.field_int_cb(g, oracle_point_field, a, b, mode == "inf", what, FINE)
        v = out[0:3] if what == 1 else out[3:6]
        assert st[4] >= 1
        tol = _tol(name, ref, 0 if "value_split" in ln else ln["prc"])
        assert np.abs(v - ref).max() < tol, (name, ln["mode"], ln["id"], v, ref)


@pytest.mark.parametrize("name", GIVEN)
def test_newton38_oracle_pinned_on_smooth_lines(rad, name):
    """The restated Newton 3/8 integral reproduces the reference's finite
    integrals on lines that cross no element."""
    h = BUILDERS[name](rad)
    g = model.pack_sources(rad._objs, h, tuple(rad._rand))
    n = 0
    for ln in GOLD["cases"][name]["lines"]:
        if ln["mode"] != "fin" or "value_split" in ln or ln["P1"] == ln["P2"]:
            continue
        what = 0 if "b" in ln["id"] else 1
        v, _ = field_int_fin(lambda P: O.field(g, P, what), ln["P1"], ln["P2"], ln["prc"])
        assert np.abs(v - np.array(ln["value"])).max() < 1e-8 + 1e-10 * np.abs(v).max()
        n += 1
    assert n >= 1


def test_infinite_integral_leaves_out_background(rad):
    """A uniform background contributes L B to a finite integral and nothing
    to an infinite one (radarccu.h:306-316)."""
    rad.UtiDelAll()
    b = rad.ObjBckg([0.1, -0.2, 0.3])
    m = rad.ObjRecMag([0, 0, 0], [2, 2, 2], [0, 0, 1])
    c = rad.ObjCnt([m, b])
    P1, P2 = [5.0, -3.0, 0.3], [5.0, 7.0, 0.3]
    g = model.pack_sources(rad._objs, c, tuple(rad._rand))
    gm = model.pack_sources(rad._objs, m, tuple(rad._rand))
    fin, _ = _native.field_int_cb(g, oracle_point_field, P1, P2, False, 1, 1e-10)
    finm, _ = _native.field_int_cb(gm, oracle_point_field, P1, P2, False, 1, 1e-10)
    assert np.allclose(fin[:3] - finm[:3], 10.0 * np.array([0.1, -0.2, 0.3]), atol=1e-9)
    inf, _ = _native.field_int_cb(g, oracle_point_field, P1, P2, True, 1, 1e-10)
    infm, _ = _native.field_int_cb(gm, oracle_point_field, P1, P2, True, 1, 1e-10)
    assert np.allclose(inf[:3], infm[:3], atol=1e-12)


def test_infinite_line_through_a_coil_is_ampere(rad):
    """Along an infinite line through the opening of a closed coil the
    integral of B is mu0 N I (the arcs' trapezoid in phi converges to it as
    the segment count grows; 20 segments: 5e-5)."""
    rad.UtiDelAll()
    rad.FldLenRndSw("off")
    ni = 10000.0
    c = rad.ObjRaceTrk([0, 0, 40], [2, 22], [60, 80], 30, 20, ni / (30 * 20), "man", "z")
    g = model.pack_sources(rad._objs, c, tuple(rad._rand))
    out, st = _native.field_int_cb(g, oracle_point_field, [10.3, 5.1, -80], [10.9, 4.7, 80], True, 1, 1e-9)
    u = np.array([0.6, -0.4, 160.0]) / np.linalg.norm([0.6, -0.4, 160.0])
    assert st[4] >= 1
    assert abs(out[:3] @ u - 4e-4 * np.pi * ni) < 1e-4 * 4e-4 * np.pi * ni


# ---------------------------------------------------------------------------
# GPU: rad.FldInt on the device field
# ---------------------------------------------------------------------------
@pytest.mark.gpu
@pytest.mark.parametrize("name", GIVEN + RELAXED)
def test_fldint_matches_reference(rad, cuda, name):
    h = BUILDERS[name](rad)
    solve = GOLD["cases"][name]["solve"]
    if solve is not None:
        rad.Solve(h, solve[0], solve[1], 4)
    rad.FldCmpCrt(1e-4, 1e-3, FINE, 1.0, 1e-5, 1e-5)
    try:
        for ln in GOLD["cases"][name]["lines"]:
            mode, a, b, ref = _target(ln)
            v = np.array(rad.FldInt(h, mode, ln["id"], a, b))
            tol = _tol(name, ref, 0 if "value_split" in ln else ln["prc"])
            assert np.abs(v - ref).max() < tol, (name, ln["mode"], ln["id"], v, ref)
    finally:
        rad.FldCmpCrt(1e-4, 1e-3, 1e-3, 1.0, 1e-5, 1e-5)


@pytest.mark.gpu
def test_fldint_component_strings_on_device(rad, cuda):
    h = BUILDERS["array_given"](rad)
    rad.FldCmpCrt(1e-4, 1e-3, FINE, 1.0, 1e-5, 1e-5)
    try:
        mode, a, b = GOLD["ids"]["line"]
        for fid, ref in GOLD["ids"]["values"].items():
            v = rad.FldInt(h, mode, fid, a, b)
            assert type(v) is type(ref), fid
            assert np.allclose(v, ref, rtol=1e-9, atol=1e-9), fid
    finally:
        rad.FldCmpCrt(1e-4, 1e-3, 1e-3, 1.0, 1e-5, 1e-5)


@pytest.mark.gpu
def test_device_and_oracle_quadrature_agree_on_tets(rad, cuda):
    """B and H integrals through and beside the tetrahedral mesh: the device
    field and the oracle field under the same quadrature."""
    h = tet_given(rad)
    g = model.pack_sources(rad._objs, h, tuple(rad._rand))
    for a, b, inf in [([-5.0, 2.9, 3.1], [10.0, 3.2, 2.7], True), ([-5.0, 2.9, 3.1], [10.0, 3.2, 2.7], False),
                      ([-4.0, 7.3, 8.1], [11.0, 7.1, 8.3], True)]:
        dev, _ = _native.field_int(g, a, b, inf, 3, 0, FINE)
        orc, _ = _native.field_int_cb(g, oracle_point_field, a, b, inf, 3, FINE)
        assert np.abs(dev - orc).max() < 1e-8 + 1e-9 * np.abs(orc).max()
