"""Generates tests/golden/golden.json from the reference Radia CPU module.

    make -f oracle/Makefile.ref REF=/root/reference -j8     # builds oracle/_ref
    python tests/golden/make_golden.py [/root/reference]

The reference is run (CPU build, FldLenRndSw('off')) on seeded models built by
tests/models.py; the script records the field and the relaxed magnetization
of each case.  It also copies the golden B values the reference's own MPI
solve regression stores (tests/_mpi_solve_reference.json of the reference,
serial CPU-assembly + CPU-relaxation column) and the known answer of the
reference's first example (a 1 mm cube, B at one point).
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle", "_ref"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

import models as MD  # noqa: E402
import radia as R  # noqa: E402
from util import leaf_magnetizations  # noqa: E402

CASES = {
    # name: (builder, kwargs, points, Solve prec, max iterations)
    "magnet_array_2x2": (MD.magnet_array, dict(nside=2, div=2), MD.magnet_array_points(6, 4), 1e-10, 1000),
    "sym_blocks": (MD.sym_blocks, {}, None, 1e-10, 1000),
    "mixed_sym": (MD.mixed_sym, {}, None, 1e-8, 3000),
    "iron_dipole_300": (MD.iron_dipole, dict(n_target=300), MD.iron_dipole_points(5), 1e-7, 3000),
    "tet_mesh_150": (MD.tet_mesh, dict(ncell=3, n_tets=150, chi=5.0), None, 1e-7, 3000),
    "thckpgn_4": (MD.thckpgn_model, {}, None, 1e-9, 3000),
}


def _points(name, pts):
    if pts is not None:
        return np.asarray(pts)
    rng = np.random.default_rng(sum(ord(c) for c in name))
    return rng.uniform(-60, 80, size=(60, 3)) + np.array([0.0137, 0.0291, 0.0413])


def main(ref_root=os.environ.get("RADIA_REFERENCE", "/root/reference")):
    out = {"provenance": "reference Radia CPU module built by oracle/Makefile.ref, FldLenRndSw('off')"}
    # known answer: reference example 1 (cube 1 mm, M = [-0.5, 1, 0.7], B at [0.52, 0.6, 0.7])
    R.UtiDelAll()
    R.FldLenRndSw("off")
    m = R.ObjRecMag([0, 0, 0], [1, 1, 1], [-0.5, 1, 0.7])
    out["example01"] = {"b": R.Fld(m, "b", [0.52, 0.6, 0.7]), "expected_approx": [0.12737, 0.028644, 0.077505]}
    cases = {}
    for name, (builder, kw, pts, prec, maxit) in CASES.items():
        res = builder(R, **kw)
        model = res[0] if isinstance(res, tuple) else res
        P = _points(name, pts)
        b0 = np.array(R.Fld(model, "b", P.tolist()))
        st = R.Solve(model, prec, maxit, 4)
        b = np.array(R.Fld(model, "b", P.tolist()))
        h = np.array(R.Fld(model, "h", P.tolist()))
        M = leaf_magnetizations(R, model)
        cases[name] = {"kwargs": kw, "prec": prec, "points": P.tolist(), "b_before": b0.tolist(),
                       "status": list(st), "b": b.tolist(), "h": h.tolist(), "M": M.tolist()}
        print(name, "iterations", st[3], "misfit", st[0])
    out["cases"] = cases
    gold = json.load(open(os.path.join(ref_root, "tests", "_mpi_solve_reference.json")))
    out["mpi_solve"] = {k: {"b": gold[k]["cpu_asm_cpu_relax"]["b"], "misfit": gold[k]["cpu_asm_cpu_relax"]["misfit"]}
                        for k in ("small", "mixed", "large")}
    out["mpi_solve_points"] = MD.MPI_SOLVE_POINTS
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(out, f)
    print("wrote", os.path.join(HERE, "golden.json"))


if __name__ == "__main__":
    main(*sys.argv[1:])
