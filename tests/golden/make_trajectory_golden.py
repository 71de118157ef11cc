"""Generates tests/golden/trajectory.json: electron trajectories computed by
the reference.

    make -f oracle/Makefile.ref REF=/root/reference -j8     # builds oracle/_ref
    python tests/golden/make_trajectory_golden.py

The reference Radia CPU module (FldLenRndSw('off')) builds seeded models from
tests/models.py, relaxes some of them, and tabulates FldPtcTrj for the
initial conditions below, once with its default integration (one fourth-order
Runge-Kutta step per interval) and once with the step-doubling control that
positive PrcCoord / PrcAngle switch on.  The y ranges have non-round ends so
that no Runge-Kutta stage lands on a block's face plane, where the reference's
field is NaN with FldLenRndSw('off').
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


def tet_given(R, seed=77):
    h, body = MD.tet_mesh(R, ncell=3, n_tets=150, chi=5.0)
    rng = np.random.default_rng(seed)
    for t in R.ObjCntStuf(body):
        R.ObjSetM(t, rng.normal(scale=0.6, size=3).tolist())
    return h


ADAPTIVE = (1e-6, 1e-8)     # PrcCoord (mm), PrcAngle (rad)
# name: (builder, Solve (prec, iterations) or None, [(E GeV, init, [y0, y1], np), ...])
CASES = {
    "array_given": (lambda R: MD.magnet_array(R, nside=2, div=2), None, [
        (0.05, [-10.3, 0.001, 8.1, -0.002], [-60.37, 60.21], 61),
        (0.02, [-17.3, 0.0, 6.4, 0.003], [-40.13, 30.29], 36)]),
    "sym_given": (MD.sym_blocks, None, [
        (0.2, [5.3, 0.01, 4.2, 0.0], [-30.17, 80.23], 56)]),
    "tet_given": (tet_given, None, [
        (0.1, [3.1, 0.0, 2.9, 0.0], [-10.07, 40.19], 51)]),
    "dipole_relaxed": (lambda R: MD.iron_dipole(R, n_target=300), (1e-7, 3000), [
        (0.3, [0.3, 0.0, 0.7, 0.0], [-200.13, 200.31], 81)]),
}


def main():
    out = {"provenance": "reference Radia CPU module built by oracle/Makefile.ref, FldLenRndSw('off')",
           "adaptive_prec": list(ADAPTIVE), "cases": {}}
    for name, (builder, solve, runs) in CASES.items():
        h = builder(R)
        if solve is not None:
            R.Solve(h, solve[0], solve[1], 4)
        rec = {"solve": solve, "runs": []}
        for E, init, lim, n in runs:
            R.FldCmpPrc("PrcCoord->-1,PrcAngle->-1")
            fixed = R.FldPtcTrj(h, E, init, lim, n)
            R.FldCmpPrc(f"PrcCoord->{ADAPTIVE[0]},PrcAngle->{ADAPTIVE[1]}")
            adaptive = R.FldPtcTrj(h, E, init, lim, n)
            R.FldCmpPrc("PrcCoord->-1,PrcAngle->-1")
            rec["runs"].append({"E": E, "init": init, "lim": lim, "np": n, "fixed": fixed, "adaptive": adaptive})
            print(name, E, "end fixed", fixed[-1], "adaptive", adaptive[-1])
        out["cases"][name] = rec
    with open(os.path.join(HERE, "trajectory.json"), "w") as f:
        json.dump(out, f)
    print("wrote", os.path.join(HERE, "trajectory.json"))


if __name__ == "__main__":
    main()
