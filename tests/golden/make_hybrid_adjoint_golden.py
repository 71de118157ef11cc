"""Generates tests/golden/hybrid_pole_fd.json: central finite differences of
a field loss in the pole thicknesses of a small hybrid undulator, computed
with the reference Radia CPU module.

    make -f oracle/Makefile.ref -j8                 # builds oracle/_ref
    python tests/golden/make_hybrid_adjoint_golden.py

Model: the hybrid undulator of tests/models.py with 4 block/pole pairs,
poles subdivided 2 x 2 x 2 (saturating MatSatIsoFrm iron), blocks 2 x 1 x 1
(anisotropic MatLin), one mirror plane.  Loss L = sum_k W_k . B(x_k) at 200
points in the gap with seeded weights W.  Pole k's z width changes by +-h
with its centre fixed (models.hybrid_undulator(pole_dz=...)); each gradient
is recorded at two steps, h and h/2, so a test can see the differences have
settled.  The reference stores its interaction matrix in FP32 and its
relaxation stalls near a misfit of 1e-8, which sets the noise of these
differences.
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

N_PAIRS = 4
POLE_DIV = (2, 2, 2)
BLOCK_DIV = (2, 1, 1)
STEPS = (2e-2, 1e-2)
N_POINTS = 200
W_SEED = 17
PREC, ITERS = 1e-9, 20000


def loss(W, pts, dz=None):
    g = MD.hybrid_undulator(R, n_pairs=N_PAIRS, pole_div=POLE_DIV, block_div=BLOCK_DIV, pole_dz=dz)[0]
    st = R.Solve(g, PREC, ITERS, 4)
    B = np.array(R.Fld(g, "b", pts.tolist()))
    return float(np.sum(B * W)), float(st[0])


def main():
    pts = MD.hybrid_points(n=N_POINTS, n_pairs=N_PAIRS)
    W = np.random.default_rng(W_SEED).normal(size=pts.shape)
    L0, m0 = loss(W, pts)
    out = {"provenance": f"reference Radia CPU module (oracle/_ref), FldLenRndSw('off'), Solve({PREC}, {ITERS}, 4)",
           "n_pairs": N_PAIRS, "pole_div": list(POLE_DIV), "block_div": list(BLOCK_DIV), "steps": list(STEPS),
           "n_points": N_POINTS, "w_seed": W_SEED, "loss": L0, "misfit": m0, "grad_dz": {}}
    for k in range(N_PAIRS):
        g = []
        for h in STEPS:
            vals = []
            for s in (1.0, -1.0):
                dz = np.zeros(N_PAIRS)
                dz[k] = s * h
                vals.append(loss(W, pts, dz)[0])
            g.append((vals[0] - vals[1]) / (2 * h))
        out["grad_dz"][str(k)] = g
        print(k, g, flush=True)
    with open(os.path.join(HERE, "hybrid_pole_fd.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
