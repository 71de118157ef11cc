"""Generates tests/golden/adjoint_fd.json: central finite differences of a
field loss computed with the reference Radia CPU module.

    make -f oracle/Makefile.ref REF=/root/reference -j8     # builds oracle/_ref
    python tests/golden/make_adjoint_golden.py

Model: the planar undulator of tests/models.py with 2 x 4 blocks, each
subdivided 2 x 2 x 2 (64 elements, anisotropic MatLin).  Loss
L = sum_k W_k . B(x_k) at 200 on-axis points with seeded weights W.  For a
few blocks the script perturbs the block remanence vector (magnetization and
MatLin easy axis together) and the block centre by +-h and records
(L(+h) - L(-h)) / 2h from the reference's own Solve (method 4) and Fld.
The reference interaction matrix is FP32, so these differences carry a small
relative noise; the tests compare with that in mind.
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

NPER = 4
H = 1e-3
BLOCKS = [0, 3, 5, 6]


def loss(W, pts, mr_off=None, c_off=None):
    g, _ = MD.undulator(R, nper_row=NPER, div=2, mr_offsets=mr_off, c_offsets=c_off)
    R.Solve(g, 1e-12, 20000, 4)
    B = np.array(R.Fld(g, "b", pts.tolist()))
    return float(np.sum(B * W))


def main():
    pts = MD.undulator_points(n=200, nper_row=NPER)
    W = np.random.default_rng(11).normal(size=pts.shape)
    nb = 2 * NPER
    out = {"provenance": "reference Radia CPU module (oracle/_ref), FldLenRndSw('off'), Solve(1e-12, 20000, 4)",
           "nper_row": NPER, "div": 2, "h": H, "n_points": int(pts.shape[0]), "w_seed": 11,
           "loss": loss(W, pts), "grad_mr": {}, "grad_c": {}}
    for b in BLOCKS:
        for a in range(3):
            for kind in ("mr", "c"):
                vals = []
                for s in (1.0, -1.0):
                    d = np.zeros((nb, 3))
                    d[b, a] = s * H
                    vals.append(loss(W, pts, mr_off=d if kind == "mr" else None, c_off=d if kind == "c" else None))
                out["grad_" + kind][f"{b},{a}"] = (vals[0] - vals[1]) / (2 * H)
    with open(os.path.join(HERE, "adjoint_fd.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
