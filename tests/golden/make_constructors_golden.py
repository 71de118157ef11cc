"""Golden vectors for a relaxed model built from ObjArcPgnMag ('sym' and
'nosym'), ObjCylMag and ObjMltExtRtg with linear anisotropic and saturating
materials, from the compiled reference module.

    make -f oracle/Makefile.ref REF=/root/reference -j8     # builds oracle/_ref
    python tests/golden/make_constructors_golden.py         # writes tests/golden/constructors.json

The reference relaxes with Solve(obj, 1e-8, 5000, 4) under FldLenRndSw('off');
the file holds its status and B at 30 seeded points.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle", "_ref"))


def build(X):
    """The model, for the reference module or radiacuda_b200.rad alike."""
    X.UtiDelAll()
    X.FldLenRndSw("off")
    arc = X.ObjArcPgnMag([0.0, 0.0], "z", [[10, -2], [14, -2], [14, 2], [10, 2]], [0.1, 1.7], 4, "nosym", [0.0, 1.0, 0.0])
    X.MatApl(arc, X.MatLin([0.06, 0.17], [0.0, 1.2, 0.1]))
    arc2 = X.ObjArcPgnMag([0.0, 0.0], "z", [[10, 5], [14, 5], [14, 8], [10, 8]], [0.1, 1.7], 4, "sym", [0.0, 1.0, 0.0])
    X.MatApl(arc2, X.MatLin([0.05, 0.15], [0.0, 1.1, 0.0]))
    cyl = X.ObjCylMag([-20.0, 3.0, 0.5], 4.0, 6.0, 10, "x", [1.0, 0.0, 0.0])
    X.MatApl(cyl, X.MatSatIsoFrm([2000, 1.5], [100, 0.4], [10, 0.2]))
    sl = X.ObjMltExtRtg([[[5, -20, -3], [6, 4]], [[5.2, -20, 0], [4, 3]], [[5, -19.8, 2.5], [6.5, 4.2]]], [0, 0, 0.5])
    X.MatApl(sl, X.MatSatIsoFrm([2000, 1.5], [100, 0.4], [10, 0.2]))
    return X.ObjCnt([arc, arc2, cyl, sl])


POINTS = (np.random.default_rng(4).uniform(-25, 20, size=(30, 3)) + np.array([0.0137, 0.0071, 0.0113])).tolist()


def main():
    import radia as R

    h = build(R)
    st = R.Solve(h, 1e-8, 5000, 4)
    B = R.Fld(h, "b", POINTS)
    with open(os.path.join(HERE, "constructors.json"), "w") as f:
        json.dump({"status": list(st), "points": POINTS, "b": B}, f)


if __name__ == "__main__":
    main()
