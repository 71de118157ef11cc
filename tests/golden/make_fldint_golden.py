"""Generates tests/golden/fldint.json: field integrals computed by the reference.

    make -f oracle/Makefile.ref REF=/root/reference -j8     # builds oracle/_ref
    python tests/golden/make_fldint_golden.py

The reference Radia CPU module (FldLenRndSw('off')) builds seeded models from
tests/models.py, relaxes some of them, and evaluates FldInt on lines chosen
to cross magnets, to run beside them, through symmetry images, background
fields and coils.  Infinite integrals of blocks and polyhedra are analytic in
the reference (radrec.cpp:468, radplnr2.cpp:390); finite ones are its Newton
3/8 sums at the PrcBInt recorded with each case.  The magnetization of every
relaxable element after the reference's relaxation is recorded too, so that
the CPU tests can evaluate the same magnetized geometry without relaxing.

Two of the reference's answers are not the field integral, and the file says
so for each line it concerns ("value_split"):
  * a finite line that crosses magnets: the per-element Newton sums stop when
    two successive sums agree to PrcBInt, which the jump of the field at the
    element's faces can satisfy early (errors of 1e-2 T mm were seen);
  * an infinite line through polyhedra: the polygon formula assumes the line
    misses the body (radexpgn.cpp:704 says so for extruded polygons);
  * an infinite line through the opening of a coil of arcs: the reference's
    arc integral (radarccu.cpp:461-700) falls short of mu0 N I (Ampere's law,
    which the reference's own finite integrals approach).
For those lines "value_split" is the reference's own FldInt 'fin' summed over
sub-segments cut at every element boundary the line crosses (each piece
smooth for every element); for an infinite line it covers the finite segment
P1 -+ "split_half" u (background fields included), which the tests integrate
as a finite line.
"""
from __future__ import annotations

import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle", "_ref"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

import models as MD  # noqa: E402
import radia as R  # noqa: E402
from util import leaf_magnetizations  # noqa: E402


def tet_given(R, seed=77):
    """150-tet mesh with seeded magnetizations (no relaxation), background on."""
    h, body = MD.tet_mesh(R, ncell=3, n_tets=150, chi=5.0)
    rng = np.random.default_rng(seed)
    for t in R.ObjCntStuf(body):
        R.ObjSetM(t, rng.normal(scale=0.6, size=3).tolist())
    return h


def leaf_handles(R, h):
    out = []
    for x in R.ObjCntStuf(h):
        sub = R.ObjCntStuf(x)
        if not sub or sub == [x]:
            out.append(x)
        else:
            out.extend(leaf_handles(R, x))
    return out


def box_crossings(R, h, p1, p2, mirrors=False):
    """Line parameters (0..1) where p1 -> p2 enters / leaves each leaf box
    (and, with mirrors, its images in the planes x = 0 and z = 0)."""
    p1, p2 = np.asarray(p1, float), np.asarray(p2, float)
    d = p2 - p1
    ts = []
    boxes = []
    for lf in leaf_handles(R, h):
        lim = np.array(R.ObjGeoLim(lf)).reshape(3, 2)
        boxes.append(lim)
        if mirrors:
            mx = lim.copy()
            mx[0] = -lim[0, ::-1]
            mz = lim.copy()
            mz[2] = -lim[2, ::-1]
            mxz = mx.copy()
            mxz[2] = -lim[2, ::-1]
            boxes += [mx, mz, mxz]
    for lim in boxes:
        t0, t1 = -np.inf, np.inf
        for k in range(3):
            if d[k] == 0:
                if not (lim[k, 0] <= p1[k] <= lim[k, 1]):
                    t0, t1 = 1, 0
                continue
            a, b = sorted(((lim[k, 0] - p1[k]) / d[k], (lim[k, 1] - p1[k]) / d[k]))
            t0, t1 = max(t0, a), min(t1, b)
        if t1 > t0:
            ts += [t0, t1]
    return ts


def tet_crossings(p1, p2):
    """Line parameters where p1 -> p2 enters / leaves each tetrahedron of the
    150-tet mesh (vertices as tests/models.py makes them)."""
    p1, p2 = np.asarray(p1, float), np.asarray(p2, float)
    d = p2 - p1
    ts = []
    for v in MD.tet_mesh_vertices(3, 150):
        c = v.mean(axis=0)
        t0, t1 = -np.inf, np.inf
        for f in MD.TET_FACES:
            a, b, e = v[f[0] - 1], v[f[1] - 1], v[f[2] - 1]
            n = np.cross(b - a, e - a)
            if n @ (c - a) > 0:
                n = -n
            A, B = n @ (p1 - a), n @ d      # inside: A + B t <= 0
            if B > 0:
                t1 = min(t1, -A / B)
            elif B < 0:
                t0 = max(t0, -A / B)
            elif A > 0:
                t0, t1 = 1, 0
        if t1 > t0:
            ts += [t0, t1]
    return ts


def _piece(R, h, fid, q1, q2, depth=0):
    """Reference finite integral over one smooth piece.  A Newton point on the
    face plane of an element the piece does not cross (NaN with FldLenRndSw
    off) is avoided by cutting the piece at an irrational fraction."""
    v = np.array(R.FldInt(h, "fin", fid, q1.tolist(), q2.tolist()))
    if np.all(np.isfinite(v)):
        return v
    if depth >= 6:
        raise RuntimeError(f"reference FldInt not finite on {q1} -> {q2}")
    m = q1 + 0.41421356237 * (q2 - q1)
    return _piece(R, h, fid, q1, m, depth + 1) + _piece(R, h, fid, m, q2, depth + 1)


def split_integral(R, h, fid, p1, p2, ts, prc):
    """Sum of the reference's finite integrals over the pieces of p1 -> p2."""
    p1, p2 = np.asarray(p1, float), np.asarray(p2, float)
    cuts = []
    for t in sorted({0.0, 1.0} | {t for t in ts if 0.0 < t < 1.0}):
        if not cuts or t - cuts[-1] > 1e-12:    # faces shared by neighbours: one cut
            cuts.append(t)
    cuts[-1] = 1.0
    R.FldCmpCrt(1e-4, 1e-3, prc, 1.0, 1e-5, 1e-5)
    tot = np.zeros(3)
    # each piece stops GAP mm short of the cuts: the reference's Newton points
    # include the ends, and on a face plane its field is NaN (FldLenRndSw off),
    # within 1e-10 mm of a pole face it overflows.  Each gap half is added
    # back by the midpoint rule on its own side of the cut (error ~ GAP^3 B'').
    L = np.linalg.norm(p2 - p1)
    eps = GAP / L
    comp = "b" if "b" in fid.lower() else "h"
    for a, b in zip(cuts[:-1], cuts[1:]):
        a, b = (a + eps if a > 0 else a), (b - eps if b < 1 else b)
        if b - a < 1e-12:
            continue
        q1, q2 = (p1 + a * (p2 - p1)).tolist(), (p1 + b * (p2 - p1)).tolist()
        tot += _piece(R, h, fid, np.array(q1), np.array(q2))
    inner = [t for t in cuts if 0.0 < t < 1.0]
    if inner:
        mids = [p1 + (t + sgn * 0.5 * eps) * (p2 - p1) for t in inner for sgn in (-1.0, 1.0)]
        tot += GAP * np.array(R.Fld(h, comp, [m.tolist() for m in mids])).sum(axis=0)
    return tot.tolist()


def array_given(R):
    return MD.magnet_array(R, nside=2, div=2)


def undulator_small(R):
    return MD.undulator(R, nper_row=8, div=1)[0]


# name: (builder, Solve (prec, max iterations) or None, lines)
# line: (mode, id, P1, P2, PrcBInt)
FINE = 1e-9
SPLIT_HALF = 400.0
GAP = 1e-6
CASES = {
    "array_given": (array_given, None, [
        ("inf", "ib", [-17.3, -40.0, 1.1], [-17.3, 40.0, 1.3], FINE),        # through two blocks
        ("inf", "ih", [-17.3, -40.0, 1.1], [-17.3, 40.0, 1.3], FINE),
        ("inf", "ib", [-40.0, -12.2, 8.5], [40.0, -12.0, 8.7], FINE),        # beside the blocks
        ("fin", "ib", [-40.0, -12.2, 8.5], [25.0, -12.0, 8.7], FINE),
        ("fin", "ib", [-25.0, -17.3, 1.1], [5.0, -16.1, 0.7], 1e-6, "boxes"),  # crossing, finite
        ("fin", "ih", [-25.0, -17.3, 1.1], [5.0, -16.1, 0.7], 1e-6, "boxes"),
        ("fin", "ib", [-3.1, -14.2, 2.0], [-3.1, -14.2, 2.0], FINE),          # zero length
    ]),
    "array_relaxed": (array_given, (1e-10, 1000), [
        ("inf", "ib", [-17.3, -40.0, 1.1], [-17.3, 40.0, 1.3], FINE),
        ("fin", "ib", [-40.0, -12.2, 8.5], [25.0, -12.0, 8.7], FINE),
    ]),
    "tet_given": (tet_given, None, [
        ("inf", "ib", [-5.0, 2.9, 3.1], [10.0, 3.2, 2.7], FINE, "tets"),     # through the mesh
        ("inf", "ih", [-5.0, 2.9, 3.1], [10.0, 3.2, 2.7], FINE, "tets"),
        ("fin", "ib", [-4.0, 7.3, 8.1], [11.0, 7.1, 8.3], FINE),             # outside (background L B)
        ("inf", "ib", [-4.0, 7.3, 8.1], [11.0, 7.1, 8.3], FINE),
        ("fin", "ib", [-5.0, 2.9, 3.1], [10.0, 3.2, 2.7], 1e-6, "tets"),     # crossing, finite
    ]),
    "tet_relaxed": (lambda R: MD.tet_mesh(R, ncell=3, n_tets=150, chi=5.0)[0], (1e-7, 3000), [
        ("inf", "ib", [-4.0, 7.3, 8.1], [11.0, 7.1, 8.3], FINE),
        ("fin", "ib", [-4.0, 7.3, 8.1], [11.0, 7.1, 8.3], FINE),
    ]),
    "sym_given": (MD.sym_blocks, None, [
        ("inf", "ib", [-40.0, 6.1, 4.3], [40.0, 6.6, 4.1], FINE),            # through mirrored images
        ("inf", "ib", [1.3, -10.0, -2.2], [1.9, 70.0, 1.7], FINE),           # through the rotated block
        ("fin", "ib", [-45.0, 20.3, 15.7], [45.0, 19.1, 16.2], FINE),
    ]),
    "dipole_relaxed": (lambda R: MD.iron_dipole(R, n_target=300), (1e-7, 3000), [
        ("inf", "ib", [0.31, -60.0, 0.73], [0.29, 60.0, 0.77], FINE),        # through the gap, coil around
        ("fin", "ib", [0.31, -150.0, 0.73], [0.29, 150.0, 0.77], FINE),
        # through both poles and the coil opening: the reference's infinite
        # integral of the arcs misses part of mu0 N I here (Ampere)
        ("inf", "ib", [10.3, 5.1, -80.0], [10.9, 4.7, 80.0], FINE, "mirrored boxes"),
    ]),
    "undulator_given": (undulator_small, None, [
        # on the axis; the ends are off the block face planes z = 5 k (the
        # reference's Newton points would land on them, where it returns NaN)
        ("inf", "ib", [0.13, 0.07, -60.3], [0.13, 0.07, 59.9], FINE),
        ("fin", "ib", [0.13, 0.07, -60.3], [0.13, 0.07, 59.9], FINE),
    ]),
}

# component strings evaluated on one line (OutFieldIntCompRes layouts)
ID_LINE = ("inf", [-17.3, -40.0, 1.1], [-17.3, 40.0, 1.3])
IDS = ["", "i", "ib", "ibx", "iby", "ibz", "ih", "ihx", "ihz", "ibxibz", "ibyihx", "bz", "IBY", "h", "ix"]


def main():
    out = {"provenance": "reference Radia CPU module built by oracle/Makefile.ref, FldLenRndSw('off')",
           "cases": {}}
    for name, (builder, solve, lines) in CASES.items():
        h = builder(R)
        if solve is not None:
            R.Solve(h, solve[0], solve[1], 4)
        rec = {"solve": solve, "M": leaf_magnetizations(R, h).tolist(), "lines": []}
        for mode, fid, p1, p2, prc, *split in lines:
            R.FldCmpCrt(1e-4, 1e-3, prc, 1.0, 1e-5, 1e-5)
            t0 = time.time()
            v = R.FldInt(h, mode, fid, p1, p2)
            dt = time.time() - t0
            entry = {"mode": mode, "id": fid, "P1": p1, "P2": p2, "prc": prc, "value": v}
            if split:
                a, b = np.asarray(p1, float), np.asarray(p2, float)
                if mode == "inf":
                    u = (b - a) / np.linalg.norm(b - a)
                    a, b = a - SPLIT_HALF * u, a + SPLIT_HALF * u
                    entry["split_half"] = SPLIT_HALF
                ts = (tet_crossings(a, b) if split[0] == "tets"
                      else box_crossings(R, h, a, b, mirrors=split[0] == "mirrored boxes"))
                entry["value_split"] = split_integral(R, h, fid, a, b, ts, FINE)
                entry["split_pieces"] = len(ts)
                print(f"{'':16s} split over {len(ts)} crossings: {entry['value_split']}")
            rec["lines"].append(entry)
            print(f"{name:16s} {mode} {fid:4s} prc {prc:.0e}: {v}  ({dt:.2f} s)")
        out["cases"][name] = rec
    # component layouts on array_given
    h = array_given(R)
    R.FldCmpCrt(1e-4, 1e-3, FINE, 1.0, 1e-5, 1e-5)
    out["ids"] = {"line": list(ID_LINE),
                  "values": {fid: R.FldInt(h, ID_LINE[0], fid, ID_LINE[1], ID_LINE[2]) for fid in IDS}}
    with open(os.path.join(HERE, "fldint.json"), "w") as f:
        json.dump(out, f, indent=0)
    print("wrote", os.path.join(HERE, "fldint.json"))


if __name__ == "__main__":
    main()
