"""Golden vectors for ObjMltExtPgn and ObjMltExtRtg from the compiled reference module.

    make -f oracle/Makefile.ref REF=/root/reference -j8     # builds oracle/_ref
    python tests/golden/make_mltextpgn_golden.py            # writes tests/golden/mltextpgn.json

For each case: the slices, the magnetization, the reference's piece count
(0 for a single polyhedron, else the container size) and B at 40 seeded
points plus 2 fixed ones, with FldLenRndSw('off').  The cases are the
polyhedral sphere of the reference's example 4 (15 slices of 15-gons between
two poles, M = [1, 0, 0]: B inside is about 2/3 T) and shapes for the piece
rules: a waist (two pieces), a prism of three equal slices (a flat crease,
two pieces), two crossed segments (a tetrahedron), a square to a segment
(a wedge) and a pole above two hexagons (a cone).  Attitudes increase in
every case; with decreasing attitudes the reference builds a different solid.
"""
import json
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle", "_ref"))


def sphere_slices(r, nphi, nz):
    """Slices of a sphere of radius r: nz - 1 inner nphi-gons between two poles."""
    dz = 2.0 * r / nz
    z = -r + dz
    dphi = 2.0 * math.pi / nphi
    out = [[[[0.0, 0.0]], -r]]
    for _ in range(1, nz):
        ct = math.cos(math.asin(z / r))
        out.append([[[r * math.cos(k * dphi) * ct, r * math.sin(k * dphi) * ct] for k in range(nphi)], z])
        z += dz
    out.append([[[0.0, 0.0]], r])
    return out


def cases():
    hexa = [[0, -2], [1.7, -1], [1.7, 1], [0, 2], [-1.7, 1], [-1.7, -1]]
    return {
        "example04_sphere": (sphere_slices(1.0, 15, 15), [1.0, 0.0, 0.0]),
        "waist": ([[[[-2, -2], [2, -2], [2, 2], [-2, 2]], 0.0], [[[-0.5, -0.5], [0.5, -0.5], [0.5, 0.5], [-0.5, 0.5]], 1.3],
                   [[[-2, -1.5], [2.2, -2], [2, 2], [-2, 2.1]], 2.9]], [0.3, -0.2, 1.1]),
        "prism_flat_crease": ([[[[0, 0], [3, 0], [0, 2]], 0.0], [[[0, 0], [3, 0], [0, 2]], 1.0], [[[0, 0], [3, 0], [0, 2]], 2.0]],
                              [0.0, 1.0, 0.0]),
        "crossed_segments": ([[[[0, 0], [4, 0]], 0.0], [[[1, -1], [1, 1]], 2.0]], [0.5, 0.5, 0.5]),
        "square_to_segment": ([[[[-1, -1], [1, -1], [1, 1], [-1, 1]], -1.0], [[[-0.8, 0.0], [0.8, 0.0]], 0.7]], [1.0, 0.0, 0.0]),
        "cone": ([[[[0.5 * x, 0.5 * y] for x, y in hexa], -1.0], [hexa, 3.0], [[[0.0, 0.0]], 7.5]], [0.0, 0.0, 1.0]),
    }


def rectangle_cases():
    """ObjMltExtRtg layers [[x, y, z], [wx, wy]]: a three-layer frustum and a waist."""
    return {
        "rtg_frustum": ([[[0.1, 0.2, 0.0], [4.0, 3.0]], [[0.3, 0.1, 2.0], [2.0, 1.5]], [[0.2, 0.3, 3.5], [0.6, 0.4]]],
                        [0.2, 0.4, 1.0]),
        "rtg_waist": ([[[0.0, 0.0, 0.0], [4.0, 4.0]], [[0.2, 0.0, 1.2], [1.0, 1.2]], [[0.0, 0.1, 2.5], [4.4, 3.9]]],
                      [1.0, 0.0, 0.3]),
    }


def main():
    import radia as R

    rng = np.random.default_rng(3)
    out = {}
    for name, (sl, M) in cases().items():
        R.UtiDelAll()
        R.FldLenRndSw("off")
        h = R.ObjMltExtPgn(sl, M)
        P = rng.uniform(-3.0, 3.0, size=(40, 3)) + np.array([0.0137, 0.0071, 1.2])
        P = np.vstack([P, [[0.001, 0.0007, 0.0013], [0.0123, 0.0211, 2.0137]]])
        B = np.array(R.Fld(h, "b", P.tolist()))
        out[name] = {"slices": sl, "M": M, "pieces": int(R.ObjCntSize(h)), "points": P.tolist(), "b": B.tolist()}
    rng = np.random.default_rng(8)
    for name, (layers, M) in rectangle_cases().items():
        R.UtiDelAll()
        R.FldLenRndSw("off")
        h = R.ObjMltExtRtg(layers, M)
        P = rng.uniform(-3.0, 3.0, size=(30, 3)) + np.array([0.0137, 0.0071, 1.5])
        B = np.array(R.Fld(h, "b", P.tolist()))
        out[name] = {"layers": layers, "M": M, "pieces": int(R.ObjCntSize(h)), "points": P.tolist(), "b": B.tolist()}
    with open(os.path.join(HERE, "mltextpgn.json"), "w") as f:
        json.dump(out, f)


if __name__ == "__main__":
    main()
